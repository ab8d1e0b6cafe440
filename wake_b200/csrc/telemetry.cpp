// Host-side telemetry arithmetic in FP64.
//
// Strouhal frequency of a lift history, restating the reference's analyser
// (src/forces/strouhal_analyzer.cpp:39-84): mean removal, Hann window over the
// first min(n, 4096) samples, zero padding to a power of two (capped at 4096),
// radix-2 FFT, and the peak power bin at index >= 1. The reference computes in
// float; this computes in double.
#include <cmath>
#include <complex>
#include <cstddef>
#include <vector>

#include "wake_gpu.h"

namespace {

void fft_inplace(std::vector<std::complex<double>>& a) {
    const std::size_t n = a.size();
    for (std::size_t i = 1, j = 0; i < n; ++i) {
        std::size_t bit = n >> 1;
        while (j & bit) {
            j ^= bit;
            bit >>= 1;
        }
        j ^= bit;
        if (i < j) std::swap(a[i], a[j]);
    }
    const double pi = 3.141592653589793238462643383279502884;
    for (std::size_t len = 2; len <= n; len <<= 1) {
        const std::size_t half = len / 2;
        for (std::size_t k = 0; k < half; ++k) {
            const double ang = -2.0 * pi * static_cast<double>(k) / static_cast<double>(len);
            const std::complex<double> w(std::cos(ang), std::sin(ang));
            for (std::size_t i = 0; i < n; i += len) {
                const std::complex<double> u = a[i + k], v = a[i + k + half] * w;
                a[i + k] = u + v;
                a[i + k + half] = u - v;
            }
        }
    }
}

}  // namespace

extern "C" double wake_strouhal_frequency(const double* signal, int n, double dt) {
    if (!signal || n < 16 || !(dt > 0.0)) return 0.0;
    double mean = 0.0;
    for (int i = 0; i < n; ++i) mean += signal[i];
    mean /= static_cast<double>(n);
    std::size_t len = 1;
    while (len < static_cast<std::size_t>(n)) len <<= 1;
    if (len > 4096) len = 4096;
    const std::size_t used = std::min<std::size_t>(len, static_cast<std::size_t>(n));
    std::vector<std::complex<double>> a(len, {0.0, 0.0});
    const double pi = 3.141592653589793238462643383279502884;
    for (std::size_t i = 0; i < used; ++i) {
        const double w = 0.5 * (1.0 - std::cos(2.0 * pi * static_cast<double>(i) / static_cast<double>(used - 1)));
        a[i] = {(signal[i] - mean) * w, 0.0};
    }
    fft_inplace(a);
    std::size_t peak = 1;
    double best = 0.0;
    for (std::size_t i = 1; i < len / 2; ++i) {
        const double p = std::norm(a[i]);
        if (p > best) {
            best = p;
            peak = i;
        }
    }
    return static_cast<double>(peak) / (static_cast<double>(len) * dt);
}
