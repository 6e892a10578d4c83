// iqfile.cu -- SDRIQ001 snapshots (internal/iqfile/iqfile.go): write, memory-
// mapped read, and a looping replay source that delivers blocks straight
// into host or device buffers for the runner.
//
// File layout (little-endian): magic "SDRIQ001", sample rate int64, centre
// frequency float64, sample count int64, then count x {re, im} float32.
#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <fcntl.h>
#include <new>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>

#include <cuda_runtime.h>

#include "../../include/gpudemod.h"

namespace {
constexpr char kMagic[8] = {'S', 'D', 'R', 'I', 'Q', '0', '0', '1'};
constexpr size_t kHeader = 32;
}  // namespace

struct gpud_iqfile {
    int fd = -1;
    void *map = nullptr;
    size_t map_bytes = 0;
    const gpud_float2 *iq = nullptr;
    gpud_iqfile_meta meta{};
    int64_t pos = 0;          // next sample delivered (wraps at the end)
    bool registered = false;  // the mapping is page-locked for DMA
    bool reg_tried = false;
};

// Write (iqfile.go:33-59).
GPUD_API int GPUD_CALL gpud_iqfile_write(const char *path, const gpud_float2 *iq, int64_t n, int64_t sample_rate,
                                         double center_hz) {
    if (!path || n < 0 || (n > 0 && !iq)) return GPUD_E_ARG;
    FILE *f = std::fopen(path, "wb");
    if (!f) return GPUD_E_IO;
    unsigned char hdr[kHeader];
    std::memcpy(hdr, kMagic, 8);
    uint64_t sr = (uint64_t)sample_rate, cnt = (uint64_t)n, cb;
    std::memcpy(&cb, &center_hz, 8);
    for (int b = 0; b < 8; ++b) {  // explicit little-endian
        hdr[8 + b] = (unsigned char)(sr >> (8 * b));
        hdr[16 + b] = (unsigned char)(cb >> (8 * b));
        hdr[24 + b] = (unsigned char)(cnt >> (8 * b));
    }
    bool ok = std::fwrite(hdr, 1, kHeader, f) == kHeader;
    // the samples: float32 pairs in the host's (little-endian) byte order
    if (ok && n > 0) ok = std::fwrite(iq, sizeof(gpud_float2), (size_t)n, f) == (size_t)n;
    ok = (std::fclose(f) == 0) && ok;
    return ok ? 0 : GPUD_E_IO;
}

// Read / NewSource (iqfile.go:62-116): the samples stay in the page cache and
// are mapped, not copied; a bad magic or a short file is an error.
GPUD_API int GPUD_CALL gpud_iqfile_open(const char *path, gpud_iqfile **out, gpud_iqfile_meta *meta) {
    if (!path || !out) return GPUD_E_ARG;
    *out = nullptr;
    int fd = ::open(path, O_RDONLY);
    if (fd < 0) return GPUD_E_IO;
    struct stat st;
    if (::fstat(fd, &st) != 0 || (size_t)st.st_size < kHeader) {
        ::close(fd);
        return GPUD_E_FORMAT;
    }
    unsigned char hdr[kHeader];
    if (::pread(fd, hdr, kHeader, 0) != (ssize_t)kHeader || std::memcmp(hdr, kMagic, 8) != 0) {
        ::close(fd);
        return GPUD_E_FORMAT;
    }
    uint64_t sr = 0, cb = 0, cnt = 0;
    for (int b = 0; b < 8; ++b) {
        sr |= (uint64_t)hdr[8 + b] << (8 * b);
        cb |= (uint64_t)hdr[16 + b] << (8 * b);
        cnt |= (uint64_t)hdr[24 + b] << (8 * b);
    }
    if (cnt > ((uint64_t)st.st_size - kHeader) / 8) {  // fewer samples on disk than the header says
        ::close(fd);
        return GPUD_E_FORMAT;
    }
    auto *f = new (std::nothrow) gpud_iqfile();
    if (!f) {
        ::close(fd);
        return GPUD_E_ARG;
    }
    f->fd = fd;
    f->meta.sample_rate = (int64_t)sr;
    std::memcpy(&f->meta.center_hz, &cb, 8);
    f->meta.samples = (int64_t)cnt;
    f->map_bytes = kHeader + (size_t)cnt * 8;
    f->map = ::mmap(nullptr, f->map_bytes, PROT_READ, MAP_SHARED, fd, 0);
    if (f->map == MAP_FAILED) {
        f->map = nullptr;
        ::close(fd);
        delete f;
        return GPUD_E_IO;
    }
    f->iq = reinterpret_cast<const gpud_float2 *>(static_cast<const char *>(f->map) + kHeader);
    if (meta) *meta = f->meta;
    *out = f;
    return 0;
}

GPUD_API void GPUD_CALL gpud_iqfile_close(gpud_iqfile *f) {
    if (!f) return;
    if (f->registered) cudaHostUnregister(f->map);
    if (f->map) ::munmap(f->map, f->map_bytes);
    if (f->fd >= 0) ::close(f->fd);
    delete f;
}

// Source.ReadIQ (iqfile.go:128-148): the next n samples, looping at the end
// of the file (an empty file gives zeros), into a host buffer or, with
// dst_on_device, a device buffer on `stream` (one copy up to the end of the
// file and one after each wrap).
GPUD_API int GPUD_CALL gpud_iqfile_read(gpud_iqfile *f, gpud_float2 *dst, int64_t n, int dst_on_device,
                                        void *stream) {
    if (!f || n < 0 || (n > 0 && !dst)) return GPUD_E_ARG;
    if (n == 0) return 0;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int64_t len = f->meta.samples;
    if (len == 0) {
        if (dst_on_device) return cudaMemsetAsync(dst, 0, (size_t)n * 8, s) == cudaSuccess ? 0 : GPUD_E_CUDA;
        std::memset(dst, 0, (size_t)n * 8);
        return 0;
    }
    if (dst_on_device && !f->reg_tried) {
        // page-locked mapping: device copies DMA straight from the page cache
        f->reg_tried = true;
        f->registered = cudaHostRegister(f->map, f->map_bytes, cudaHostRegisterReadOnly) == cudaSuccess;
        if (!f->registered) cudaGetLastError();
    }
    int64_t done = 0;
    while (done < n) {
        const int64_t take = std::min<int64_t>(n - done, len - f->pos);
        if (dst_on_device) {
            if (cudaMemcpyAsync(dst + done, f->iq + f->pos, (size_t)take * 8, cudaMemcpyHostToDevice, s) !=
                cudaSuccess)
                return GPUD_E_CUDA;
        } else {
            std::memcpy(dst + done, f->iq + f->pos, (size_t)take * 8);
        }
        done += take;
        f->pos += take;
        if (f->pos >= len) f->pos = 0;
    }
    return 0;
}

GPUD_API int GPUD_CALL gpud_iqfile_seek(gpud_iqfile *f, int64_t pos) {
    if (!f || pos < 0 || (f->meta.samples > 0 && pos >= f->meta.samples) || (f->meta.samples == 0 && pos != 0))
        return GPUD_E_ARG;
    f->pos = pos;
    return 0;
}

GPUD_API int64_t GPUD_CALL gpud_iqfile_tell(const gpud_iqfile *f) { return f ? f->pos : -1; }
