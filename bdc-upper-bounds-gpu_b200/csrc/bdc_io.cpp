// bdc_io.cpp -- the reference's two file formats and the error string.
//
//   cache_n_k      backend/cache_io.h:7-44 (name, raw uint32 write/read);
//                  this reader also checks the size (the reference reads
//                  whatever is there, and try_to_open_file exits on a
//                  missing file, backend/utils.cc:46-53)
//   dist_n_k.txt   backend/main_BAA.cu:3-18 (read: whitespace separated
//                  doubles), 84-91 / 113-119 (write "%.17g\n"); written here
//                  through a temporary file and rename so that an
//                  interrupted save never truncates the only checkpoint
#include <cerrno>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>

#include "../../include/bdc_b200.h"

namespace bdc {

static thread_local std::string g_last_error;

void set_last_error(const char* fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_last_error = buf;
}

const char* last_error() { return g_last_error.c_str(); }

}  // namespace bdc

extern "C" {

const char* bdc_last_error(void) { return bdc::last_error(); }

bdc_status bdc_read_cache_file(const char* path, int n, int k, uint32_t* out) {
    if (!path || !out || n < 0 || k < 0 || n + k > 40) {
        bdc::set_last_error("bdc_read_cache_file: bad arguments");
        return BDC_ERR_ARG;
    }
    FILE* f = fopen(path, "rb");
    if (!f) {
        bdc::set_last_error("failed to open file %s (%s)", path, strerror(errno));
        return BDC_ERR_IO;
    }
    const size_t want = (size_t)1 << (n + k);
    size_t got = fread(out, sizeof(uint32_t), want, f);
    uint32_t extra;
    size_t more = fread(&extra, sizeof(uint32_t), 1, f);
    fclose(f);
    if (got != want || more != 0) {
        bdc::set_last_error("cache file %s holds %s entries, expected %zu (2^(%d+%d))", path,
                            more ? "more" : std::to_string(got).c_str(), want, n, k);
        return BDC_ERR_IO;
    }
    return BDC_OK;
}

bdc_status bdc_write_cache_file(const char* path, int n, int k, const uint32_t* data) {
    if (!path || !data || n < 0 || k < 0 || n + k > 40) {
        bdc::set_last_error("bdc_write_cache_file: bad arguments");
        return BDC_ERR_ARG;
    }
    FILE* f = fopen(path, "wb");
    if (!f) {
        bdc::set_last_error("failed to open file %s (%s)", path, strerror(errno));
        return BDC_ERR_IO;
    }
    const size_t want = (size_t)1 << (n + k);
    size_t put = fwrite(data, sizeof(uint32_t), want, f);
    int rc = fclose(f);
    if (put != want || rc != 0) {
        bdc::set_last_error("short write to %s", path);
        return BDC_ERR_IO;
    }
    return BDC_OK;
}

bdc_status bdc_read_dist_file(const char* path, double* out, int64_t cap, int64_t* count) {
    if (!path || !count) {
        bdc::set_last_error("bdc_read_dist_file: bad arguments");
        return BDC_ERR_ARG;
    }
    FILE* f = fopen(path, "r");
    if (!f) {
        bdc::set_last_error("Could not open %s for reading (%s)", path, strerror(errno));
        return BDC_ERR_IO;
    }
    int64_t c = 0;
    double v;
    while (fscanf(f, "%lf", &v) == 1) {
        if (out) {
            if (c >= cap) {
                fclose(f);
                bdc::set_last_error("%s holds more than %lld values", path, (long long)cap);
                return BDC_ERR_IO;
            }
            out[c] = v;
        }
        ++c;
    }
    int bad = !feof(f);
    fclose(f);
    if (bad) {
        bdc::set_last_error("%s: value %lld is not a number", path, (long long)c + 1);
        return BDC_ERR_IO;
    }
    *count = c;
    return BDC_OK;
}

bdc_status bdc_write_dist_file(const char* path, const double* p, int64_t count) {
    if (!path || (!p && count > 0) || count < 0) {
        bdc::set_last_error("bdc_write_dist_file: bad arguments");
        return BDC_ERR_ARG;
    }
    std::string tmp = std::string(path) + ".tmp";
    FILE* f = fopen(tmp.c_str(), "w");
    if (!f) {
        bdc::set_last_error("failed to open file %s (%s)", tmp.c_str(), strerror(errno));
        return BDC_ERR_IO;
    }
    for (int64_t i = 0; i < count; ++i) {
        if (fprintf(f, "%.17g\n", p[i]) < 0) {
            fclose(f);
            remove(tmp.c_str());
            bdc::set_last_error("short write to %s", tmp.c_str());
            return BDC_ERR_IO;
        }
    }
    if (fclose(f) != 0 || rename(tmp.c_str(), path) != 0) {
        remove(tmp.c_str());
        bdc::set_last_error("could not replace %s (%s)", path, strerror(errno));
        return BDC_ERR_IO;
    }
    return BDC_OK;
}

}  // extern "C"
