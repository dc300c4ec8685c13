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

// ------------------------------------------------------- observable streams
// A per-sweep (or per-flip) series of FP64 observables on disk, for offline
// autocorrelation analysis (umc_tau_int) of runs longer than memory.  Layout,
// little-endian as the host writes it:
//   char magic[8] "UMCOBS01"; uint32 version (1); uint32 columns;
//   uint64 records; uint64 seed; uint64 first (counter of record 0);
//   int32 model; uint32 reserved; double beta;          -- 56 bytes
//   char names[columns][32] (NUL-padded column names);
//   double data[records][columns].
// `records` is rewritten after every append, so a stream cut short by a crash
// still reads back every record its header counts.

#include <cstdio>
#include <cstring>
#include <string>

namespace {
constexpr char kObsMagic[8] = {'U', 'M', 'C', 'O', 'B', 'S', '0', '1'};
constexpr uint32_t kObsName = 32;

struct ObsHeader
{
    char magic[8];
    uint32_t version, columns;
    uint64_t records, seed, first;
    int32_t model;
    uint32_t reserved;
    double beta;
};
static_assert(sizeof(ObsHeader) == 56, "observable stream header layout");

ObsHeader read_header(std::FILE* f, const char* path)
{
    ObsHeader h{};
    if (std::fread(&h, sizeof h, 1, f) != 1 || std::memcmp(h.magic, kObsMagic, 8) != 0 || h.version != 1 ||
        h.columns == 0)
        throw umc::Error(UMC_ERR_INVALID_ARGUMENT, std::string("not an observable stream: ") + path);
    return h;
}
}  // namespace

struct umc_obs_stream
{
    std::FILE* f = nullptr;
    ObsHeader h{};
};

extern "C" {

int umc_obs_stream_create(const char* path, uint32_t columns, const char* const* names, uint64_t seed,
                          uint64_t first, int32_t model, double beta, umc_obs_stream** out)
{
    return umc::sguard([&] {
        if (!path || !out) throw umc::Error(UMC_ERR_INVALID_ARGUMENT, "null argument");
        if (columns == 0 || columns > 4096) throw umc::Error(UMC_ERR_INVALID_ARGUMENT, "1 to 4096 columns");
        auto* s = new umc_obs_stream;
        s->f = std::fopen(path, "w+b");
        if (!s->f) {
            delete s;
            throw umc::Error(UMC_ERR_INVALID_ARGUMENT, std::string("cannot create ") + path);
        }
        std::memcpy(s->h.magic, kObsMagic, 8);
        s->h.version = 1;
        s->h.columns = columns;
        s->h.seed = seed;
        s->h.first = first;
        s->h.model = model;
        s->h.beta = beta;
        std::vector<char> nm(size_t(columns) * kObsName, 0);
        for (uint32_t c = 0; names && c < columns; ++c)
            if (names[c]) std::strncpy(nm.data() + size_t(c) * kObsName, names[c], kObsName - 1);
        const bool ok = std::fwrite(&s->h, sizeof s->h, 1, s->f) == 1 && std::fwrite(nm.data(), 1, nm.size(), s->f) == nm.size();
        if (!ok || std::fflush(s->f) != 0) {
            std::fclose(s->f);
            delete s;
            throw umc::Error(UMC_ERR_INVALID_ARGUMENT, std::string("cannot write ") + path);
        }
        *out = s;
    });
}

int umc_obs_stream_append(umc_obs_stream* s, const double* records, uint64_t n)
{
    return umc::sguard([&] {
        if (!s || (n && !records)) throw umc::Error(UMC_ERR_INVALID_ARGUMENT, "null argument");
        if (n == 0) return;
        const long data = long(sizeof(ObsHeader) + size_t(s->h.columns) * kObsName);
        const uint64_t vals = n * s->h.columns;
        if (std::fseek(s->f, data + long(s->h.records * s->h.columns * sizeof(double)), SEEK_SET) != 0 ||
            std::fwrite(records, sizeof(double), vals, s->f) != vals)
            throw umc::Error(UMC_ERR_INVALID_ARGUMENT, "observable stream: write failed");
        s->h.records += n;
        if (std::fflush(s->f) != 0 || std::fseek(s->f, 0, SEEK_SET) != 0 || std::fwrite(&s->h, sizeof s->h, 1, s->f) != 1 ||
            std::fflush(s->f) != 0)
            throw umc::Error(UMC_ERR_INVALID_ARGUMENT, "observable stream: header update failed");
    });
}

int umc_obs_stream_close(umc_obs_stream* s)
{
    return umc::sguard([&] {
        if (!s) return;
        const int rc = std::fclose(s->f);
        delete s;
        if (rc != 0) throw umc::Error(UMC_ERR_INVALID_ARGUMENT, "observable stream: close failed");
    });
}

int umc_obs_stream_info(const char* path, uint32_t* columns, uint64_t* records, uint64_t* seed, uint64_t* first,
                        int32_t* model, double* beta, char* names)
{
    return umc::sguard([&] {
        if (!path) throw umc::Error(UMC_ERR_INVALID_ARGUMENT, "null path");
        std::FILE* f = std::fopen(path, "rb");
        if (!f) throw umc::Error(UMC_ERR_INVALID_ARGUMENT, std::string("cannot open ") + path);
        try {
            const ObsHeader h = read_header(f, path);
            if (columns) *columns = h.columns;
            if (records) *records = h.records;
            if (seed) *seed = h.seed;
            if (first) *first = h.first;
            if (model) *model = h.model;
            if (beta) *beta = h.beta;
            if (names && std::fread(names, 1, size_t(h.columns) * kObsName, f) != size_t(h.columns) * kObsName)
                throw umc::Error(UMC_ERR_INVALID_ARGUMENT, "observable stream: truncated names");
        } catch (...) {
            std::fclose(f);
            throw;
        }
        std::fclose(f);
    });
}

int umc_obs_stream_read(const char* path, uint64_t first_record, uint64_t n, double* out)
{
    return umc::sguard([&] {
        if (!path || (n && !out)) throw umc::Error(UMC_ERR_INVALID_ARGUMENT, "null argument");
        std::FILE* f = std::fopen(path, "rb");
        if (!f) throw umc::Error(UMC_ERR_INVALID_ARGUMENT, std::string("cannot open ") + path);
        try {
            const ObsHeader h = read_header(f, path);
            if (first_record > h.records || n > h.records - first_record)
                throw umc::Error(UMC_ERR_OUT_OF_RANGE, "observable stream: records beyond the stream");
            const long at = long(sizeof h + size_t(h.columns) * kObsName + first_record * h.columns * sizeof(double));
            const uint64_t vals = n * h.columns;
            if (std::fseek(f, at, SEEK_SET) != 0 || std::fread(out, sizeof(double), vals, f) != vals)
                throw umc::Error(UMC_ERR_INVALID_ARGUMENT, "observable stream: truncated data");
        } catch (...) {
            std::fclose(f);
            throw;
        }
        std::fclose(f);
    });
}

}  // extern "C"
