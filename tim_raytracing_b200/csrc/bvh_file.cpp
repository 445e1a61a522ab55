// bvh_file.cpp -- versioned on-disk form of an uploaded scene (include/tim_rt.h,
// tim_rt_bvh_file_*): the fillGpuBuffer bytes with their seven ranges and push
// constants (src/Renderer/BVHBuilder.cpp:1319-1534, BVHData.cpp:43-48) and the
// BVHGeometry vertex arrays (src/Renderer/BVHGeometry.cpp:69-78), so a scene
// built once (the reference builder is not deterministic in its threaded mode,
// BVHBuilder.cpp:851-894) is traced from identical bytes on every run.
//
// Layout, little-endian:
//   header (160 B): magic "TIMRTBVH", version, header size, blob size, ranges,
//                   push constants, aabb, vertex counts, section bits, reserved
//   blob (padded to 16 B), positions (12 B per vertex), normals and uvs when the
//   section bits say so (12 / 8 B per vertex),
//   trailer: FNV-1a 64 of every byte before it.
// Reading checks the magic, version, sizes against the file length, the checksum
// and then the BVH itself (validate_bvh, as tim_rt_upload_bvh does).
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <vector>
#include "tim_rt.h"
#include "internal.h"

using timrt::set_error;
using timrt::validate_bvh;

namespace {

constexpr char kMagic[8] = {'T', 'I', 'M', 'R', 'T', 'B', 'V', 'H'};
constexpr uint32_t kVersion = 1, kHeaderBytes = 160;
constexpr uint32_t kHasNormals = 1u, kHasUvs = 2u;

struct FileHeader {
    char magic[8];
    uint32_t version, header_bytes;
    uint64_t blob_bytes;
    uint32_t ranges[7][2];
    tim_rt_push_constants pc;
    float aabb[6];
    uint32_t num_vertex, max_vertex, sections;
    uint8_t reserved[160 - 8 - 8 - 8 - 56 - 20 - 24 - 12];
};
static_assert(sizeof(FileHeader) == kHeaderBytes, "header layout");

inline uint64_t pad16(uint64_t x) { return (x + 15ull) & ~15ull; }

struct Fnv {
    uint64_t h = 1469598103934665603ull;
    void add(const void* p, uint64_t n) {
        const uint8_t* b = static_cast<const uint8_t*>(p);
        for (uint64_t i = 0; i < n; ++i) {
            h ^= b[i];
            h *= 1099511628211ull;
        }
    }
};

uint64_t payload_bytes(const FileHeader& h) {
    const uint64_t nv = h.num_vertex;
    return pad16(h.blob_bytes) + 12 * nv + ((h.sections & kHasNormals) ? 12 * nv : 0) +
           ((h.sections & kHasUvs) ? 8 * nv : 0);
}

}  // namespace

struct tim_rt_bvh_file {
    FileHeader h{};
    std::vector<uint8_t> data;   // payload
    const uint8_t* blob() const { return data.data(); }
    const float* pos() const { return reinterpret_cast<const float*>(data.data() + pad16(h.blob_bytes)); }
    const float* nrm() const { return (h.sections & kHasNormals) ? pos() + 3ull * h.num_vertex : nullptr; }
    const float* uv() const {
        if (!(h.sections & kHasUvs)) return nullptr;
        return pos() + 3ull * h.num_vertex * ((h.sections & kHasNormals) ? 2 : 1);
    }
};

extern "C" {

int tim_rt_bvh_file_write(const char* path, const void* bvh_bytes, uint64_t n_bytes, const uint32_t ranges[7][2],
                          const tim_rt_push_constants* pc, const float aabb[6], const float* pos, const float* nrm,
                          const float* uv, uint32_t max_vertex, uint32_t num_vertex) {
    if (!path || !bvh_bytes || !ranges || !pc || !pos || num_vertex == 0) {
        set_error("tim_rt_bvh_file_write: null argument or no vertices");
        return TIM_RT_EINVAL;
    }
    std::string err;
    uint32_t depth = 0;
    if (!validate_bvh(static_cast<const uint8_t*>(bvh_bytes), n_bytes, ranges, pc->numNodes, num_vertex, pc->numLights,
                      pc->numBlas, &depth, err)) {
        set_error("tim_rt_bvh_file_write: " + err);
        return TIM_RT_EINVAL;
    }
    FileHeader h{};
    std::memcpy(h.magic, kMagic, 8);
    h.version = kVersion;
    h.header_bytes = kHeaderBytes;
    h.blob_bytes = n_bytes;
    std::memcpy(h.ranges, ranges, sizeof(h.ranges));
    h.pc = *pc;
    if (aabb) std::memcpy(h.aabb, aabb, sizeof(h.aabb));
    h.num_vertex = num_vertex;
    h.max_vertex = max_vertex < num_vertex ? num_vertex : max_vertex;
    h.sections = (nrm ? kHasNormals : 0u) | (uv ? kHasUvs : 0u);
    const std::string tmp = std::string(path) + ".tmp";
    std::FILE* f = std::fopen(tmp.c_str(), "wb");
    if (!f) {
        set_error(std::string("tim_rt_bvh_file_write: cannot open ") + tmp);
        return TIM_RT_EINVAL;
    }
    Fnv fnv;
    bool ok = true;
    auto put = [&](const void* p, uint64_t n) {
        if (!ok || n == 0) return;
        fnv.add(p, n);
        ok = std::fwrite(p, 1, n, f) == n;
    };
    static const uint8_t zeros[16] = {};
    put(&h, sizeof(h));
    put(bvh_bytes, n_bytes);
    put(zeros, pad16(n_bytes) - n_bytes);
    put(pos, 12ull * num_vertex);
    if (nrm) put(nrm, 12ull * num_vertex);
    if (uv) put(uv, 8ull * num_vertex);
    const uint64_t sum = fnv.h;
    if (ok) ok = std::fwrite(&sum, 1, 8, f) == 8;
    ok = (std::fclose(f) == 0) && ok;
    if (!ok || std::rename(tmp.c_str(), path) != 0) {
        std::remove(tmp.c_str());
        set_error(std::string("tim_rt_bvh_file_write: write failed for ") + path);
        return TIM_RT_EINVAL;
    }
    return TIM_RT_OK;
}

int tim_rt_bvh_file_read(const char* path, tim_rt_bvh_file** out) {
    if (!path || !out) {
        set_error("tim_rt_bvh_file_read: null argument");
        return TIM_RT_EINVAL;
    }
    *out = nullptr;
    std::unique_ptr<std::FILE, int (*)(std::FILE*)> f(std::fopen(path, "rb"), &std::fclose);
    if (!f) {
        set_error(std::string("tim_rt_bvh_file_read: cannot open ") + path);
        return TIM_RT_EINVAL;
    }
    std::fseek(f.get(), 0, SEEK_END);
    const long len = std::ftell(f.get());
    std::fseek(f.get(), 0, SEEK_SET);
    auto file = std::make_unique<tim_rt_bvh_file>();
    FileHeader& h = file->h;
    const std::string who = std::string("tim_rt_bvh_file_read: ") + path + ": ";
    if (len < (long)(kHeaderBytes + 8) || std::fread(&h, 1, sizeof(h), f.get()) != sizeof(h) ||
        std::memcmp(h.magic, kMagic, 8) != 0) {
        set_error(who + "not a BVH file");
        return TIM_RT_EINVAL;
    }
    if (h.version != kVersion || h.header_bytes != kHeaderBytes) {
        set_error(who + "unsupported version " + std::to_string(h.version));
        return TIM_RT_EUNSUPPORTED;
    }
    const uint64_t want = payload_bytes(h);
    if (h.num_vertex == 0 || (uint64_t)len != kHeaderBytes + want + 8) {
        set_error(who + "size does not match its header (truncated or corrupt)");
        return TIM_RT_EINVAL;
    }
    file->data.resize(want);
    uint64_t sum = 0;
    if (std::fread(file->data.data(), 1, want, f.get()) != want || std::fread(&sum, 1, 8, f.get()) != 8) {
        set_error(who + "read failed");
        return TIM_RT_EINVAL;
    }
    Fnv fnv;
    fnv.add(&h, sizeof(h));
    fnv.add(file->data.data(), want);
    if (fnv.h != sum) {
        set_error(who + "checksum mismatch (corrupt file)");
        return TIM_RT_EINVAL;
    }
    std::string err;
    uint32_t depth = 0;
    if (!validate_bvh(file->blob(), h.blob_bytes, h.ranges, h.pc.numNodes, h.num_vertex, h.pc.numLights, h.pc.numBlas,
                      &depth, err)) {
        set_error(who + err);
        return TIM_RT_EINVAL;
    }
    *out = file.release();
    return TIM_RT_OK;
}

int tim_rt_bvh_file_info(const tim_rt_bvh_file* f, const uint8_t** bytes, uint64_t* size, uint32_t ranges[7][2],
                         tim_rt_push_constants* pc, float aabb[6], const float** pos, const float** nrm,
                         const float** uv, uint32_t* max_vertex, uint32_t* num_vertex) {
    if (!f) {
        set_error("tim_rt_bvh_file_info: null file");
        return TIM_RT_EINVAL;
    }
    if (bytes) *bytes = f->blob();
    if (size) *size = f->h.blob_bytes;
    if (ranges) std::memcpy(ranges, f->h.ranges, sizeof(f->h.ranges));
    if (pc) *pc = f->h.pc;
    if (aabb) std::memcpy(aabb, f->h.aabb, sizeof(f->h.aabb));
    if (pos) *pos = f->pos();
    if (nrm) *nrm = f->nrm();
    if (uv) *uv = f->uv();
    if (max_vertex) *max_vertex = f->h.max_vertex;
    if (num_vertex) *num_vertex = f->h.num_vertex;
    return TIM_RT_OK;
}

void tim_rt_bvh_file_free(tim_rt_bvh_file* f) { delete f; }

int tim_rt_upload_bvh_file(tim_rt_ctx* ctx, const char* path, uint32_t flags, tim_rt_scene_id* out) {
    tim_rt_bvh_file* f = nullptr;
    int rc = tim_rt_bvh_file_read(path, &f);
    if (rc) return rc;
    rc = tim_rt_upload_bvh(ctx, f->blob(), f->h.blob_bytes, f->h.ranges, f->pos(), f->nrm(), f->uv(), f->h.max_vertex,
                           f->h.num_vertex, &f->h.pc, flags, out);
    tim_rt_bvh_file_free(f);
    return rc;
}

}  // extern "C"
