// C-ABI shim around mach's reference CUDA kernel (mach-beamform 0.1.3).
//
// The reference translation unit src/mach/kernel.cu is compiled here UNMODIFIED,
// straight from the reference tree (the build recipe puts src/mach on the include
// path); nanobind is replaced by the stand-in headers next to this file.  This
// library is a checker and a baseline only: the mach_b200 product never links it.
//
// Two entry points reach the reference's own code:
//   machref_beamform_impl     -> _beamform_impl<T>   (kernel.cu:714-891), device pointers,
//                                the path nb_beamform takes when every array is on CUDA
//   machref_beamform_binding  -> beamform<T>         (kernel.cu:1032-1209), the binding with
//                                its CPU->GPU staging, used for end-to-end timing
#include "kernel.cu"

#include <cstring>
#include <stdexcept>

namespace {

void write_error(char* err, size_t errlen, const char* msg) {
    if (err && errlen) {
        std::strncpy(err, msg, errlen - 1);
        err[errlen - 1] = '\0';
    }
}

}  // namespace

extern "C" {

int machref_beamform_impl(int is_complex, const void* d_channel, const float* d_rx,
                          const float* d_scan, const float* d_tx, void* d_out, uint32_t n_rx,
                          uint32_t n_samples, uint64_t n_vox, uint32_t n_frames, float f_number,
                          float rx_start_s, float sampling_freq_hz, float sound_speed_m_s,
                          float modulation_freq_hz, float tukey_alpha, int interp_type, char* err,
                          size_t errlen) {
    try {
        const auto interp = static_cast<InterpolationType>(interp_type);
        if (is_complex) {
            _beamform_impl<float2>(static_cast<const float2*>(d_channel),
                                   reinterpret_cast<const float3*>(d_rx),
                                   reinterpret_cast<const float3*>(d_scan), d_tx,
                                   static_cast<float2*>(d_out), n_rx, n_samples, n_vox, n_frames,
                                   f_number, rx_start_s, sampling_freq_hz, sound_speed_m_s,
                                   modulation_freq_hz, tukey_alpha, interp);
        } else {
            _beamform_impl<float>(static_cast<const float*>(d_channel),
                                  reinterpret_cast<const float3*>(d_rx),
                                  reinterpret_cast<const float3*>(d_scan), d_tx,
                                  static_cast<float*>(d_out), n_rx, n_samples, n_vox, n_frames,
                                  f_number, rx_start_s, sampling_freq_hz, sound_speed_m_s,
                                  modulation_freq_hz, tukey_alpha, interp);
        }
    } catch (const std::exception& e) {
        write_error(err, errlen, e.what());
        return -1;
    }
    return 0;
}

// Device types follow DLPack: 1 = CPU, 2 = CUDA.
int machref_beamform_binding(int is_complex, const void* channel, int dev_channel,
                             const float* rx, int dev_rx, const float* scan, int dev_scan,
                             const float* tx, int dev_tx, void* out, int dev_out, uint32_t n_rx,
                             uint32_t n_samples, uint64_t n_vox, uint32_t n_frames,
                             float f_number, float rx_start_s, float sampling_freq_hz,
                             float sound_speed_m_s, float modulation_freq_hz, float tukey_alpha,
                             int interp_type, char* err, size_t errlen) {
    try {
        const size_t ch_shape[3] = {n_rx, n_samples, n_frames};
        const size_t rx_shape[2] = {n_rx, 3};
        const size_t scan_shape[2] = {static_cast<size_t>(n_vox), 3};
        const size_t tx_shape[1] = {static_cast<size_t>(n_vox)};
        const size_t out_shape[2] = {static_cast<size_t>(n_vox), n_frames};
        nb::ndarray<const float, nb::shape<-1, 3>, nb::c_contig> a_rx(rx, 2, rx_shape, dev_rx);
        nb::ndarray<const float, nb::shape<-1, 3>, nb::c_contig> a_scan(scan, 2, scan_shape,
                                                                          dev_scan);
        nb::ndarray<const float, nb::ndim<1>, nb::c_contig> a_tx(tx, 1, tx_shape, dev_tx);
        const auto interp = static_cast<InterpolationType>(interp_type);
        if (is_complex) {
            using C = std::complex<float>;
            nb::ndarray<const C, nb::ndim<3>, nb::c_contig> a_ch(static_cast<const C*>(channel),
                                                                 3, ch_shape, dev_channel);
            nb::ndarray<C, nb::ndim<2>, nb::c_contig> a_out(static_cast<C*>(out), 2, out_shape,
                                                            dev_out);
            beamform<C>(a_ch, a_rx, a_scan, a_tx, a_out, f_number, rx_start_s, sampling_freq_hz,
                        sound_speed_m_s, modulation_freq_hz, tukey_alpha, interp);
        } else {
            nb::ndarray<const float, nb::ndim<3>, nb::c_contig> a_ch(
                static_cast<const float*>(channel), 3, ch_shape, dev_channel);
            nb::ndarray<float, nb::ndim<2>, nb::c_contig> a_out(static_cast<float*>(out), 2,
                                                                out_shape, dev_out);
            beamform<float>(a_ch, a_rx, a_scan, a_tx, a_out, f_number, rx_start_s,
                            sampling_freq_hz, sound_speed_m_s, modulation_freq_hz, tukey_alpha,
                            interp);
        }
    } catch (const std::exception& e) {
        write_error(err, errlen, e.what());
        return -1;
    }
    return 0;
}

const char* machref_last_warning(void) { return machref_warning_text().c_str(); }

const char* machref_nvcc_version(void) { return NVCC_VERSION_STR; }

}  // extern "C"
