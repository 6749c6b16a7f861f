// Transmit split of one job into launches (host code only, no CUDA).
//
// The gather kernels address one launch's channel data with 32-bit sample offsets, so a job
// whose channel data holds 2^31 samples or more runs as several launches of whole transmits,
// each below 2^31 samples.  The allocating entry points and the allocation-free one share
// this arithmetic; tests/test_split_cpu.py checks it (boundaries at 1, 2, 64 and 65 launches).
#pragma once

#include <algorithm>
#include <cstdint>

namespace mach_b200 {

constexpr int64_t kLaunchSampleLimit = (int64_t{1} << 31) - 1;  // samples per launch, at most

struct TransmitSplit {
    int64_t max_tx;    // transmits per launch (>= 1)
    int64_t n_launch;  // launches (>= 1, also for a job without transmits)
};

// per_tx = samples of one transmit (n_rx * n_samples * n_frames), n_tx = transmits of the job.
inline TransmitSplit split_transmits(int64_t per_tx, int64_t n_tx) {
    TransmitSplit s{};
    s.max_tx = std::max<int64_t>(1, kLaunchSampleLimit / std::max<int64_t>(per_tx, 1));
    s.n_launch = (std::max<int64_t>(n_tx, 1) + s.max_tx - 1) / s.max_tx;
    return s;
}

// First transmit of launch `k`, and the transmits it covers.
inline int64_t launch_first_tx(const TransmitSplit& s, int64_t k) { return k * s.max_tx; }
inline int64_t launch_tx_count(const TransmitSplit& s, int64_t n_tx, int64_t k) {
    return std::max<int64_t>(0, std::min<int64_t>(s.max_tx, n_tx - launch_first_tx(s, k)));
}

}  // namespace mach_b200
