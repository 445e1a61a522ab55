// host_fuzz.cpp -- sanitizer fuzzing of the library's host-side code paths that
// read untrusted input: the BVH image validation and the 8-wide collapse
// (csrc/bvh_layout.cpp), the BVH file reader (csrc/bvh_file.cpp) and the host
// builder (csrc/bvh_build.cpp). Built by tests/test_host_fuzz.py together with
// those sources under AddressSanitizer and UBSan; any out-of-bounds access or
// undefined behaviour aborts the run. Every input must be refused with a status
// or accepted, and every accepted image must pass tim_rt_wide_check.
//
//   host_fuzz image <file.timbvh> <seed> <count>   corrupt words of a valid image
//   host_fuzz file  <file.timbvh> <seed> <count>   corrupt headers / payloads of a file
//   host_fuzz build <seed> <count>                 build degenerate triangle soups
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <random>
#include <string>
#include <vector>
#include "tim_rt.h"
#include "internal.h"

namespace timrt {
void set_error(const std::string&) {}   // the library's error slot lives in the GPU runtime, not linked here
}
extern "C" int tim_rt_upload_bvh(tim_rt_ctx*, const void*, uint64_t, const uint32_t[7][2], const float*, const float*,
                                 const float*, uint32_t, uint32_t, const tim_rt_push_constants*, uint32_t,
                                 tim_rt_scene_id*) {
    return TIM_RT_EDEVICE;   // no GPU in this program
}

namespace {

int fail_count = 0;

struct Loaded {
    std::vector<uint8_t> bytes;
    uint32_t ranges[7][2];
    tim_rt_push_constants pc;
    std::vector<float> pos;
};

bool load(const char* path, Loaded& L) {
    tim_rt_bvh_file* f = nullptr;
    if (tim_rt_bvh_file_read(path, &f) != TIM_RT_OK) return false;
    const uint8_t* b;
    uint64_t n;
    const float* pos;
    uint32_t nv;
    tim_rt_bvh_file_info(f, &b, &n, L.ranges, &L.pc, nullptr, &pos, nullptr, nullptr, nullptr, &nv);
    L.bytes.assign(b, b + n);
    L.pos.assign(pos, pos + 3ull * nv);
    tim_rt_bvh_file_free(f);
    return true;
}

// a valid-by-validation image must collapse and check, or be refused by the check with a status
void check_accepted(const uint8_t* b, uint64_t n, const uint32_t r[7][2], const tim_rt_push_constants& pc,
                    const float* pos, uint32_t nv) {
    tim_rt_wide_report rep;
    const int rc = tim_rt_wide_check(b, n, r, &pc, pos, nv, &rep);
    if (rc != TIM_RT_OK && rc != TIM_RT_EINVAL) ++fail_count;
}

void fuzz_image(const Loaded& L, std::mt19937_64& rng, int count, long& acc, long& ref) {
    const uint32_t nv = (uint32_t)(L.pos.size() / 3);
    for (int it = 0; it < count; ++it) {
        std::vector<uint8_t> b = L.bytes;
        uint32_t r[7][2];
        std::memcpy(r, L.ranges, sizeof(r));
        tim_rt_push_constants pc = L.pc;
        const int kind = (int)(rng() % 6), flips = 1 + (int)(rng() % 4);
        for (int j = 0; j < flips; ++j) {
            if (kind <= 3) {
                const int which = kind < 2 ? TIM_RT_RANGE_NODE : TIM_RT_RANGE_LEAF;
                const uint64_t words = r[which][1] / 4;
                if (!words) continue;
                uint32_t* w = reinterpret_cast<uint32_t*>(b.data() + r[which][0]) + rng() % words;
                const uint32_t choice[] = {0u, 0xFFFFFFFFu, 0x3FFFFFFFu, 0x80000000u, 0x7FC00000u, (uint32_t)rng(),
                                           *w + 1u, *w ^ (1u << (rng() % 32))};
                *w = choice[rng() % 8];
            } else if (kind == 4) {
                pc.numNodes = (uint32_t)(rng() % (2ull * L.pc.numNodes + 2));
            } else {
                r[rng() % 7][rng() % 2] += (uint32_t)(rng() % 64) - 32u;
            }
        }
        uint32_t depth = 0;
        std::string err;
        if (timrt::validate_bvh(b.data(), b.size(), r, pc.numNodes, nv, pc.numLights, pc.numBlas, &depth, err)) {
            ++acc;
            check_accepted(b.data(), b.size(), r, pc, L.pos.data(), nv);
        } else {
            ++ref;
        }
    }
}

uint64_t fnv(const uint8_t* b, size_t n) {
    uint64_t h = 1469598103934665603ull;
    for (size_t i = 0; i < n; ++i) { h ^= b[i]; h *= 1099511628211ull; }
    return h;
}

void fuzz_file(const char* path, std::mt19937_64& rng, int count, long& acc, long& ref) {
    FILE* f = std::fopen(path, "rb");
    if (!f) { ++fail_count; return; }
    std::fseek(f, 0, SEEK_END);
    const long n = std::ftell(f);
    std::fseek(f, 0, SEEK_SET);
    std::vector<uint8_t> orig((size_t)n);
    if (std::fread(orig.data(), 1, (size_t)n, f) != (size_t)n) { std::fclose(f); ++fail_count; return; }
    std::fclose(f);
    const std::string tmp = std::string(path) + ".fuzz";
    for (int it = 0; it < count; ++it) {
        std::vector<uint8_t> b = orig;
        const int mode = (int)(rng() % 3);
        if (mode == 0) {   // header words (sizes, ranges, counts); checksum recomputed
            for (int j = 0; j < 1 + (int)(rng() % 3); ++j) {
                uint32_t* w = reinterpret_cast<uint32_t*>(b.data()) + 2 + rng() % 38;
                const uint32_t ch[] = {0u, 0xFFFFFFFFu, *w + 1u, *w - 1u, *w * 2u, (uint32_t)rng(), *w ^ (1u << (rng() % 32))};
                *w = ch[rng() % 7];
            }
        } else if (mode == 1) {   // payload words; checksum recomputed
            for (int j = 0; j < 1 + (int)(rng() % 4); ++j)
                reinterpret_cast<uint32_t*>(b.data() + 160)[rng() % ((size_t)(n - 168) / 4)] = (uint32_t)rng();
        } else {   // truncated or extended
            b.resize(rng() % 2 ? (size_t)n - 1 - rng() % 64 : (size_t)n + rng() % 64);
        }
        if (mode != 2) {
            const uint64_t h = fnv(b.data(), b.size() - 8);
            std::memcpy(b.data() + b.size() - 8, &h, 8);
        }
        FILE* g = std::fopen(tmp.c_str(), "wb");
        std::fwrite(b.data(), 1, b.size(), g);
        std::fclose(g);
        tim_rt_bvh_file* bf = nullptr;
        if (tim_rt_bvh_file_read(tmp.c_str(), &bf) == TIM_RT_OK) {
            ++acc;
            const uint8_t* bytes;
            uint64_t size;
            uint32_t r[7][2];
            tim_rt_push_constants pc;
            const float* pos;
            uint32_t nv;
            tim_rt_bvh_file_info(bf, &bytes, &size, r, &pc, nullptr, &pos, nullptr, nullptr, nullptr, &nv);
            check_accepted(bytes, size, r, pc, pos, nv);
            tim_rt_bvh_file_free(bf);
        } else {
            ++ref;
        }
    }
    std::remove(tmp.c_str());
}

void fuzz_build(std::mt19937_64& rng, int count, long& acc, long& ref) {
    std::uniform_real_distribution<float> U(0.f, 1.f);
    for (int it = 0; it < count; ++it) {
        const uint32_t nt = 1 + (uint32_t)(rng() % (rng() % 4 == 0 ? 5000 : 300));
        const int kind = (int)(rng() % 6);
        std::vector<float> pos(9ull * nt);
        for (uint32_t t = 0; t < nt; ++t)
            for (int v = 0; v < 3; ++v)
                for (int a = 0; a < 3; ++a) {
                    float x = U(rng);
                    if (kind == 1) x = 0.5f;                                    // every vertex the same point
                    if (kind == 2 && a == 2) x = 0.25f;                          // flat scene
                    if (kind == 3) x = (float)(t % 3) * 1e-30f + x * 1e-35f;    // tiny scale
                    if (kind == 4) x = x * 1e12f - 5e11f;                        // huge scale
                    if (kind == 5 && v > 0) x = pos[9ull * t + a];               // point triangles
                    pos[9ull * t + 3 * v + a] = x;
                }
        std::vector<uint32_t> rec(3ull * nt);   // one material per 21,845 triangles (16-bit local indices)
        for (uint32_t t = 0; t < nt; ++t) {
            const uint32_t chunk = t / 21845, l = 3 * (t - chunk * 21845);
            rec[3ull * t] = chunk * 21845u * 3u;
            rec[3ull * t + 1] = l | ((l + 1) << 16);
            rec[3ull * t + 2] = (l + 2) | (chunk << 16);
        }
        const uint32_t nmat = (nt + 21844) / 21845;
        std::vector<uint8_t> mats(48ull * nmat, 0);
        tim_rt_build_params p;
        tim_rt_build_params_default(&p);
        p.max_leaf_size = 1 + (uint32_t)(rng() % 8);
        tim_rt_bvh_blob* b = nullptr;
        if (tim_rt_build_bvh(pos.data(), 3 * nt, rec.data(), nt, mats.data(), nmat, nullptr, 0, &p, &b) != TIM_RT_OK) {
            ++ref;
            continue;
        }
        ++acc;
        const uint8_t* bytes;
        uint64_t size;
        uint32_t r[7][2];
        tim_rt_push_constants pc;
        float aabb[6];
        tim_rt_bvh_blob_info(b, &bytes, &size, r, &pc, aabb);
        tim_rt_wide_report rep;
        if (tim_rt_wide_check(bytes, size, r, &pc, pos.data(), 3 * nt, &rep) != TIM_RT_OK) ++fail_count;   // must pass
        tim_rt_bvh_blob_free(b);
    }
}

}  // namespace

int main(int argc, char** argv) {
    if (argc < 4) return 2;
    const std::string mode = argv[1];
    long acc = 0, ref = 0;
    if (mode == "build") {
        std::mt19937_64 rng(std::strtoull(argv[2], nullptr, 10));
        fuzz_build(rng, std::atoi(argv[3]), acc, ref);
    } else {
        if (argc < 5) return 2;
        std::mt19937_64 rng(std::strtoull(argv[3], nullptr, 10));
        if (mode == "image") {
            Loaded L;
            if (!load(argv[2], L)) return 3;
            fuzz_image(L, rng, std::atoi(argv[4]), acc, ref);
        } else if (mode == "file") {
            fuzz_file(argv[2], rng, std::atoi(argv[4]), acc, ref);
        } else {
            return 2;
        }
    }
    std::printf("accepted %ld refused %ld failures %d\n", acc, ref, fail_count);
    return fail_count ? 1 : 0;
}
