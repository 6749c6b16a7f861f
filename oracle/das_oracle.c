/*
 * FP64 C restatement of delay-and-sum beamforming, parallel over voxels with OpenMP.
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the CUDA kernels and the timed CPU
 * baseline ("port") in bench.py.  The product library never links it.
 *
 * It computes exactly what oracle/das_fp64.py computes (same rules, same
 * citations into the mach repository):
 *   aperture radius R = z / (2 f#)                    src/mach/kernel.cu:583
 *   exclusion dx^2 + dy^2 > R^2                       src/mach/kernel.cu:459-465
 *   tau = tx_arrival + |rx - voxel| / c               src/mach/kernel.cu:467-471
 *   half-Tukey weight (alpha > 0 only)                src/mach/kernel.cu:333-349, 473-482
 *   skip tau < 0 or weight == 0                       src/mach/kernel.cu:634
 *   s = (tau - t0) * fs                               src/mach/kernel.cu:637
 *   nearest / linear / quadratic bounds and taps      src/mach/kernel.cu:106-252
 *   weight * sample, then * exp(+i 2 pi f_mod tau)    src/mach/kernel.cu:649-669
 *   compounding = sum over transmits                  src/mach/experimental.py:80-97
 * with one shared deviation: nearest index == n_samples is out of bounds.
 *
 * Storage codes match include/mach_b200.h (0 f32, 1 c64, 2 f16, 3 cf16,
 * 4 bf16, 5 cbf16, 6 i16, 7 ci16).  Every sample is widened to double and
 * multiplied by `scale`.
 */
#include <math.h>
#include <stdint.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

static double half_to_double(uint16_t h) {
    /* IEEE 754 binary16 decode. */
    int sign = (h >> 15) & 1;
    int expo = (h >> 10) & 0x1f;
    int mant = h & 0x3ff;
    double v;
    if (expo == 0) {
        v = ldexp((double)mant, -24);
    } else if (expo == 31) {
        v = mant ? NAN : INFINITY;
    } else {
        v = ldexp((double)(mant | 0x400), expo - 25);
    }
    return sign ? -v : v;
}

static double bf16_to_double(uint16_t b) {
    uint32_t bits = (uint32_t)b << 16;
    float f;
    memcpy(&f, &bits, sizeof(f));
    return (double)f;
}

static int storage_is_complex(int storage) { return storage & 1; }

static size_t storage_scalar_bytes(int storage) {
    switch (storage) {
        case 0: case 1: return 4;
        default: return 2;
    }
}

/* Read scalar component `k` (0 = real/I, 1 = Q) of sample `idx` (counted in samples). */
static double load_component(int storage, const void* base, size_t idx, int k) {
    size_t comps = storage_is_complex(storage) ? 2 : 1;
    size_t pos = idx * comps + (size_t)k;
    switch (storage) {
        case 0: case 1: return (double)((const float*)base)[pos];
        case 2: case 3: return half_to_double(((const uint16_t*)base)[pos]);
        case 4: case 5: return bf16_to_double(((const uint16_t*)base)[pos]);
        default: return (double)((const int16_t*)base)[pos];
    }
}

static double tukey_weight(double r, double alpha) {
    if (r < 0.0 || r > 1.0) return 0.0;
    if (r <= 1.0 - alpha) return 1.0;
    return 0.5 - 0.5 * cos(M_PI * (1.0 - r) / alpha);
}

/*
 * out: [n_sel][n_f] doubles (real storage) or [n_sel][n_f][2] (complex storage).
 * vox_idx: optional list of n_sel voxel indices; NULL means all n_vox voxels (n_sel == n_vox).
 * Returns 0 on success, -1 on a bad argument.
 */
int das_oracle_f64(int storage, const void* channel, double scale, const float* rx,
                   const float* scan, const float* arrivals, double* out, int64_t n_tx,
                   int64_t n_rx, int64_t n_s, int64_t n_f, int64_t n_vox, const int64_t* vox_idx,
                   int64_t n_sel, double f_number, double t0, double fs, double c, double fmod,
                   double alpha, int interp, int n_threads) {
    if (storage < 0 || storage > 7 || interp < 0 || interp > 2) return -1;
    if (!vox_idx && n_sel != n_vox) return -1;
    const int cplx = storage_is_complex(storage);
    const int rotate = cplx && fmod != 0.0;
    const int comps = cplx ? 2 : 1;
    const size_t esz = storage_scalar_bytes(storage) * (size_t)comps;
    (void)esz;
#ifdef _OPENMP
    if (n_threads > 0) omp_set_num_threads(n_threads);
#else
    (void)n_threads;
#endif

#pragma omp parallel for schedule(dynamic, 16)
    for (int64_t i = 0; i < n_sel; ++i) {
        const int64_t v = vox_idx ? vox_idx[i] : i;
        double* o = out + (size_t)i * (size_t)n_f * (size_t)comps;
        for (int64_t f = 0; f < n_f * comps; ++f) o[f] = 0.0;
        const double vx = scan[3 * v + 0], vy = scan[3 * v + 1], vz = scan[3 * v + 2];
        const double radius = vz / (2.0 * f_number);
        const double radius_sq = radius * radius;
        for (int64_t e = 0; e < n_rx; ++e) {
            const double dx = (double)rx[3 * e + 0] - vx;
            const double dy = (double)rx[3 * e + 1] - vy;
            const double dz = (double)rx[3 * e + 2] - vz;
            const double h2 = dx * dx + dy * dy;
            if (h2 > radius_sq) continue;
            const double dist = sqrt(h2 + dz * dz);
            const double weight = alpha > 0.0 ? tukey_weight(sqrt(h2) / radius, alpha) : 1.0;
            if (weight == 0.0) continue;
            for (int64_t t = 0; t < n_tx; ++t) {
                const double tau = (double)arrivals[t * n_vox + v] + dist / c;
                if (tau < 0.0) continue;
                const double s = (tau - t0) * fs;
                const size_t row = ((size_t)t * (size_t)n_rx + (size_t)e) * (size_t)n_s * (size_t)n_f;
                int64_t taps[3];
                double tw[3];
                int ntap = 0;
                if (interp == 0) {
                    if (!(s >= -0.5 && s <= (double)n_s - 0.5)) continue;
                    const int64_t idx = (int64_t)nearbyint(s);
                    if (idx >= n_s) continue;
                    taps[0] = idx < 0 ? 0 : idx;
                    tw[0] = 1.0;
                    ntap = 1;
                } else if (interp == 1) {
                    if (!(s >= 0.0 && s <= (double)(n_s - 1))) continue;
                    const int64_t i0 = (int64_t)floor(s);
                    const int64_t i1 = (int64_t)ceil(s);
                    const double a = s - (double)i0;
                    taps[0] = i0;
                    taps[1] = i1;
                    tw[0] = 1.0 - a;
                    tw[1] = a;
                    ntap = 2;
                } else {
                    if (!(s >= 1.0 && s <= (double)n_s - 2.0)) continue;
                    const int64_t cc = (int64_t)nearbyint(s);
                    const double x = s - (double)cc;
                    taps[0] = cc - 1;
                    taps[1] = cc;
                    taps[2] = cc + 1;
                    tw[0] = 0.5 * x * (x - 1.0);
                    tw[1] = (1.0 - x) * (1.0 + x);
                    tw[2] = 0.5 * x * (x + 1.0);
                    ntap = 3;
                }
                double cph = 1.0, sph = 0.0;
                if (rotate) {
                    const double phi = 2.0 * M_PI * fmod * tau;
                    cph = cos(phi);
                    sph = sin(phi);
                }
                const double g = weight * scale;
                for (int64_t f = 0; f < n_f; ++f) {
                    double re = 0.0, im = 0.0;
                    if (interp == 1) {
                        /* a + t (b - a), the form of the reference's lerp */
                        const size_t ia = (row + (size_t)taps[0] * (size_t)n_f + (size_t)f);
                        const size_t ib = (row + (size_t)taps[1] * (size_t)n_f + (size_t)f);
                        const double ar = load_component(storage, channel, ia, 0);
                        const double br = load_component(storage, channel, ib, 0);
                        re = ar + tw[1] * (br - ar);
                        if (cplx) {
                            const double ai = load_component(storage, channel, ia, 1);
                            const double bi = load_component(storage, channel, ib, 1);
                            im = ai + tw[1] * (bi - ai);
                        }
                    } else {
                        for (int k = 0; k < ntap; ++k) {
                            const size_t ik = row + (size_t)taps[k] * (size_t)n_f + (size_t)f;
                            re += tw[k] * load_component(storage, channel, ik, 0);
                            if (cplx) im += tw[k] * load_component(storage, channel, ik, 1);
                        }
                    }
                    re *= g;
                    im *= g;
                    if (cplx) {
                        o[2 * f + 0] += re * cph - im * sph;
                        o[2 * f + 1] += im * cph + re * sph;
                    } else {
                        o[f] += re;
                    }
                }
            }
        }
    }
    return 0;
}

int das_oracle_max_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
