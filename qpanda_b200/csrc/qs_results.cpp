// qs_results.cpp - the reference's result formats, written from the device
// state: the .fullstate text and .fullstate.binary files of the command line
// (QPandaSDK/QuantumCommandControl/QCommand.cpp:402-480) and the outcome text
// of QPandaSDK::getResult (QPandaSDK/QPandaAPI/QPandaAPI.cpp:220-238).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <string>
#include <vector>

#include "qs_common.cuh"

namespace {

constexpr size_t kChunk = 1u << 20;              // amplitudes per device-to-host copy

struct File {
    FILE *f = nullptr;
    ~File() { if (f) fclose(f); }
};

}  // namespace

extern "C" int qs_write_fullstate(qs_state *s, const char *path_prefix, int binary)
{
    int r = qs_check_state(s);
    if (r) return r;
    if (!path_prefix || !*path_prefix) return qs_fail(QS_ERR_ARG, "qs_write_fullstate: empty path");
    if (binary != 0 && binary != 1) return qs_fail(QS_ERR_ARG, "qs_write_fullstate: binary must be 0 or 1");
    const std::string path = std::string(path_prefix) + (binary ? ".fullstate.binary" : ".fullstate");
    File out;
    out.f = fopen(path.c_str(), binary ? "wb" : "w");
    if (!out.f) return qs_fail(QS_ERR_IO, "qs_write_fullstate: cannot open %s", path.c_str());
    const size_t es = s->dtype == QS_C64 ? 8 : 16;
    std::vector<char> raw(std::min<uint64_t>(kChunk, s->N) * es);
    std::vector<double> wide(std::min<uint64_t>(kChunk, s->N) * 2);
    std::string text;
    char line[160];
    for (uint64_t base = 0; base < s->N; base += kChunk) {
        const size_t cnt = (size_t)std::min<uint64_t>(kChunk, s->N - base);
        QS_CUDA_TRY(cudaMemcpyAsync(raw.data(), static_cast<const char *>(s->amp) + base * es, cnt * es,
                                    cudaMemcpyDeviceToHost, s->stream));
        QS_CUDA_TRY(cudaStreamSynchronize(s->stream));
        if (s->dtype == QS_C64) {
            const float *f = reinterpret_cast<const float *>(raw.data());
            for (size_t i = 0; i < 2 * cnt; ++i) wide[i] = (double)f[i];
        } else {
            std::copy_n(reinterpret_cast<const double *>(raw.data()), 2 * cnt, wide.data());
        }
        if (binary) {
            if (fwrite(wide.data(), sizeof(double), 2 * cnt, out.f) != 2 * cnt)
                return qs_fail(QS_ERR_IO, "qs_write_fullstate: write to %s failed", path.c_str());
            continue;
        }
        text.clear();
        for (size_t i = 0; i < cnt; ++i) {
            // "%g" is the default formatting of a double on a C++ stream
            const unsigned long long k = (unsigned long long)(base + i);
            const int len = snprintf(line, sizeof(line), "state[%llu].real = %g state[%llu].imag = %g\n", k,
                                     wide[2 * i], k, wide[2 * i + 1]);
            text.append(line, (size_t)len);
        }
        if (fwrite(text.data(), 1, text.size(), out.f) != text.size())
            return qs_fail(QS_ERR_IO, "qs_write_fullstate: write to %s failed", path.c_str());
    }
    if (fflush(out.f) != 0) return qs_fail(QS_ERR_IO, "qs_write_fullstate: write to %s failed", path.c_str());
    return QS_OK;
}

extern "C" int qs_format_outcomes(const uint64_t *keys, const double *values, size_t count, int width, char *buf,
                                  size_t cap, size_t *needed)
{
    if (!needed) return qs_fail(QS_ERR_ARG, "qs_format_outcomes: null length output");
    if (count && (!keys || !values)) return qs_fail(QS_ERR_ARG, "qs_format_outcomes: null input");
    if (width < 1 || width > 64) return qs_fail(QS_ERR_ARG, "qs_format_outcomes: width %d", width);
    std::vector<size_t> ord(count);
    for (size_t i = 0; i < count; ++i) {
        ord[i] = i;
        if (width < 64 && (keys[i] >> width))
            return qs_fail(QS_ERR_ARG, "qs_format_outcomes: key %llu does not fit %d bits",
                           (unsigned long long)keys[i], width);
    }
    std::sort(ord.begin(), ord.end(), [&](size_t a, size_t b) { return keys[a] < keys[b]; });
    std::string text;
    char num[64];
    for (size_t k = 0; k < count; ++k) {
        const size_t i = ord[k];
        if (k && keys[ord[k - 1]] == keys[i])
            return qs_fail(QS_ERR_ARG, "qs_format_outcomes: duplicate key %llu", (unsigned long long)keys[i]);
        for (int b = width - 1; b >= 0; --b) text.push_back(((keys[i] >> b) & 1) ? '1' : '0');
        const int len = snprintf(num, sizeof(num), " %g\n", values[i]);
        text.append(num, (size_t)len);
    }
    *needed = text.size() + 1;
    if (buf) {
        if (cap < text.size() + 1) return qs_fail(QS_ERR_ARG, "qs_format_outcomes: buffer of %zu bytes, %zu needed",
                                                  cap, text.size() + 1);
        std::copy(text.begin(), text.end(), buf);
        buf[text.size()] = 0;
    }
    return QS_OK;
}
