// umc_stats.cpp -- integrated autocorrelation times and binned error bars for
// observable series (no reference counterpart: the reference's tests compare
// chain means with fixed tolerances, test/model_check.cpp:171-222).
//
// tau_int with Sokal's automatic window: with the normalised autocorrelation
// rho(t) = C(t)/C(0), tau(W) = 1/2 + sum_{t=1..W} rho(t), and W the smallest
// window with W >= c * tau(W) (Madras & Sokal 1988; c = 5 to 6 is customary).
// The statistical error of tau follows the Madras-Sokal estimate
// sqrt(2 (2W + 1) / n) * tau.  C(t) is computed directly in FP64, O(n W).
//
// Binning: the series is cut into bins of b consecutive values; the standard
// error of the mean from the bin means grows with b until bins decorrelate,
// where it equals sqrt(2 tau var / n).

#include <cmath>
#include <vector>

#include "umc_tables.hpp"

namespace umc {
namespace {

template <class F>
int sguard(F&& f)
{
    try {
        set_last_error("");
        f();
        return UMC_OK;
    } catch (const Error& e) {
        set_last_error(e.what());
        return e.code;
    } catch (const std::exception& e) {
        set_last_error(e.what());
        return UMC_ERR_INVALID_ARGUMENT;
    }
}

}  // namespace
}  // namespace umc

extern "C" {

int umc_tau_int(const double* x, uint64_t n, double c, double* tau, double* tau_err, uint64_t* window)
{
    return umc::sguard([&] {
        if (!x || n < 4) throw umc::Error(UMC_ERR_INVALID_ARGUMENT, "tau_int needs at least 4 values");
        if (!(c > 0.0)) c = 6.0;
        double mean = 0.0;
        for (uint64_t i = 0; i < n; ++i) mean += x[i];
        mean /= double(n);
        std::vector<double> d(n);
        for (uint64_t i = 0; i < n; ++i) d[i] = x[i] - mean;
        double c0 = 0.0;
        for (uint64_t i = 0; i < n; ++i) c0 += d[i] * d[i];
        c0 /= double(n);
        double t = 0.5;
        uint64_t W = 0;
        if (c0 > 0.0) {
            const uint64_t wmax = n / 2;
            for (uint64_t w = 1; w <= wmax; ++w) {
                double ct = 0.0;
                for (uint64_t i = 0; i + w < n; ++i) ct += d[i] * d[i + w];
                ct /= double(n - w);
                t += ct / c0;
                W = w;
                if (double(w) >= c * t) break;
            }
        }
        if (tau) *tau = t;
        if (tau_err) *tau_err = t * std::sqrt(2.0 * (2.0 * double(W) + 1.0) / double(n));
        if (window) *window = W;
    });
}

int umc_tau_int_multi(const double* x, uint64_t series, uint64_t length, double c, double* tau, double* tau_err,
                      uint64_t* window)
{
    return umc::sguard([&] {
        if (!x || series == 0 || length < 4) throw umc::Error(UMC_ERR_INVALID_ARGUMENT, "need series of at least 4 values");
        if (!(c > 0.0)) c = 6.0;
        // each series centred on its own mean; autocovariances pooled over series
        std::vector<double> d(series * length);
        for (uint64_t s = 0; s < series; ++s) {
            double m = 0.0;
            for (uint64_t i = 0; i < length; ++i) m += x[s * length + i];
            m /= double(length);
            for (uint64_t i = 0; i < length; ++i) d[s * length + i] = x[s * length + i] - m;
        }
        auto cov = [&](uint64_t t) {
            double a = 0.0;
            for (uint64_t s = 0; s < series; ++s) {
                const double* r = d.data() + s * length;
                for (uint64_t i = 0; i + t < length; ++i) a += r[i] * r[i + t];
            }
            return a / double(series * (length - t));
        };
        const double c0 = cov(0);
        double t = 0.5;
        uint64_t W = 0;
        if (c0 > 0.0) {
            for (uint64_t w = 1; w <= length / 2; ++w) {
                t += cov(w) / c0;
                W = w;
                if (double(w) >= c * t) break;
            }
        }
        if (tau) *tau = t;
        if (tau_err) *tau_err = t * std::sqrt(2.0 * (2.0 * double(W) + 1.0) / double(series * length));
        if (window) *window = W;
    });
}

int umc_binning_error(const double* x, uint64_t n, uint64_t bin, double* mean, double* err)
{
    return umc::sguard([&] {
        if (!x || n == 0 || bin == 0) throw umc::Error(UMC_ERR_INVALID_ARGUMENT, "empty series or zero bin");
        const uint64_t nb = n / bin;
        if (nb < 2) throw umc::Error(UMC_ERR_INVALID_ARGUMENT, "fewer than two bins");
        std::vector<double> m(nb, 0.0);
        for (uint64_t b = 0; b < nb; ++b) {
            for (uint64_t i = 0; i < bin; ++i) m[b] += x[b * bin + i];
            m[b] /= double(bin);
        }
        double mu = 0.0;
        for (double v : m) mu += v;
        mu /= double(nb);
        double var = 0.0;
        for (double v : m) var += (v - mu) * (v - mu);
        var /= double(nb - 1);
        if (mean) *mean = mu;
        if (err) *err = std::sqrt(var / double(nb));
    });
}

}  // extern "C"
