/*
 * oracle/refglsl/glsl_shim.h -- TEST INFRASTRUCTURE ONLY.
 *
 * The GLSL 4.50 language subset the reference's compute shaders use, written as
 * C++20, so that mechanically rewritten copies of those shaders (produced by
 * make_refglsl.py into oracle/_ref/glsl/, never committed) compile on the host
 * and serve as a second, independent oracle next to oracle/reftrace.c.
 *
 * Semantics chosen where GLSL leaves freedom (the same choices as reftrace.c and
 * the CUDA kernels, so that agreement tests the restatement, not the choices):
 *   - IEEE binary32 arithmetic, no FMA contraction (-ffp-contract=off), correctly
 *     rounded division and sqrt;
 *   - min / max are C99 fmin / fmax (NaN operands give the other operand);
 *   - dot() sums left to right, cross() in the textbook component order,
 *     length(v) = sqrt(dot(v, v)), normalize(v) = v / length(v), mix(x, y, a) =
 *     x * (1 - a) + y * a, clamp(x, lo, hi) = min(max(x, lo), hi);
 *   - out-of-range buffer reads return zero and out-of-range writes are dropped
 *     (Vulkan robustBufferAccess2);
 *   - rgba16f images store with round-to-nearest-even.
 * Scalar implicit conversions follow GLSL: int -> uint -> float.
 */
#pragma once
#include <cmath>
#include <cstdint>
#include <cstring>
#include <type_traits>
#include <utility>
#undef M_PI /* the reference declares its own `const float M_PI` */

namespace glsl {

typedef uint32_t uint;

/* ---------------------------------------------------------------- scalars */
template <class A> inline constexpr bool is_num_v = std::is_arithmetic_v<A> && !std::is_same_v<A, bool>;
template <class A, class B>
using promote_t = std::conditional_t<std::is_floating_point_v<A> || std::is_floating_point_v<B>, float,
                                     std::conditional_t<std::is_unsigned_v<A> || std::is_unsigned_v<B>, uint, int>>;

template <class T> inline T smin(T a, T b) {
    if constexpr (std::is_floating_point_v<T>) return std::fmin(a, b);
    else return b < a ? b : a;
}
template <class T> inline T smax(T a, T b) {
    if constexpr (std::is_floating_point_v<T>) return std::fmax(a, b);
    else return a < b ? b : a;
}
template <class A, class B, class = std::enable_if_t<is_num_v<A> && is_num_v<B>>>
inline promote_t<A, B> min(A a, B b) { using T = promote_t<A, B>; return smin<T>(T(a), T(b)); }
template <class A, class B, class = std::enable_if_t<is_num_v<A> && is_num_v<B>>>
inline promote_t<A, B> max(A a, B b) { using T = promote_t<A, B>; return smax<T>(T(a), T(b)); }
template <class A, class B, class C, class = std::enable_if_t<is_num_v<A> && is_num_v<B> && is_num_v<C>>>
inline promote_t<promote_t<A, B>, C> clamp(A x, B lo, C hi) {
    using T = promote_t<promote_t<A, B>, C>;
    return smin<T>(smax<T>(T(x), T(lo)), T(hi));
}
inline float abs(float x) { return std::fabs(x); }
inline int abs(int x) { return x < 0 ? -x : x; }
inline float sqrt(float x) { return std::sqrt(x); }
inline float pow(float x, float y) { return std::pow(x, y); }
inline float floor(float x) { return std::floor(x); }
inline float fract(float x) { return x - std::floor(x); }
inline float mod(float x, float y) { return x - y * std::floor(x / y); }
inline float sin(float x) { return std::sin(x); }
inline float cos(float x) { return std::cos(x); }
inline float acos(float x) { return std::acos(x); }
inline float exp(float x) { return std::exp(x); }
inline float sign(float x) { return x > 0.0f ? 1.0f : (x < 0.0f ? -1.0f : 0.0f); }
inline float mix(float x, float y, float a) { return x * (1.0f - a) + y * a; }
inline float step(float edge, float x) { return x < edge ? 0.0f : 1.0f; }
inline uint floatBitsToUint(float f) { uint u; std::memcpy(&u, &f, 4); return u; }
inline int floatBitsToInt(float f) { int u; std::memcpy(&u, &f, 4); return u; }
inline float uintBitsToFloat(uint u) { float f; std::memcpy(&f, &u, 4); return f; }

/* ---------------------------------------------------------------- vectors */
template <class T, int N> struct tvec;

/* A swizzle view (.xy, .xyz, .zw, .rgb ...) over the storage of a vector: reads
 * convert to a vector, writes scatter into the selected components. */
template <class T, int N, int... I> struct swz {
    T d[N];
    using V = tvec<T, (int)sizeof...(I)>;
    operator V() const { return V(d[I]...); }
    swz& operator=(const V& v) { int k = 0; ((d[I] = v.v[k++]), ...); return *this; }
    swz& operator=(const swz& o) { return *this = V(o); }
    swz& operator+=(const V& v) { return *this = V(*this) + v; }
    swz& operator-=(const V& v) { return *this = V(*this) - v; }
    swz& operator*=(const V& v) { return *this = V(*this) * v; }
};

template <class U, class T> inline constexpr bool implicit_conv_v =
    std::is_same_v<U, T> || (std::is_same_v<U, int> && !std::is_same_v<T, bool>) ||
    (std::is_same_v<U, uint> && std::is_same_v<T, float>);

#define GLSL_VEC_COMMON(N)                                                                                   \
    tvec(const tvec& o) { for (int i = 0; i < N; ++i) v[i] = o.v[i]; }                                       \
    tvec& operator=(const tvec& o) { for (int i = 0; i < N; ++i) v[i] = o.v[i]; return *this; }             \
    template <class U> explicit(!implicit_conv_v<U, T>) tvec(const tvec<U, N>& o) {                          \
        for (int i = 0; i < N; ++i) v[i] = T(o.v[i]);                                                        \
    }                                                                                                        \
    T& operator[](int i) { return v[i]; }                                                                    \
    const T& operator[](int i) const { return v[i]; }

template <class T> struct tvec<T, 2> {
    union {
        T v[2];
        struct { T x, y; };
        struct { T r, g; };
        swz<T, 2, 0, 1> xy;
        swz<T, 2, 1, 0> yx;
    };
    tvec() : v{T(0), T(0)} {}
    tvec(T a, T b) : v{a, b} {}
    explicit tvec(T s) : v{s, s} {}
    GLSL_VEC_COMMON(2)
};

template <class T> struct tvec<T, 3> {
    union {
        T v[3];
        struct { T x, y, z; };
        struct { T r, g, b; };
        swz<T, 3, 0, 1> xy;
        swz<T, 3, 0, 2> xz;
        swz<T, 3, 1, 2> yz;
        swz<T, 3, 0, 1, 2> xyz;
        swz<T, 3, 0, 1, 2> rgb;
    };
    tvec() : v{T(0), T(0), T(0)} {}
    tvec(T a, T b, T c) : v{a, b, c} {}
    explicit tvec(T s) : v{s, s, s} {}
    tvec(const tvec<T, 2>& a, T c) : v{a.v[0], a.v[1], c} {}
    explicit tvec(const tvec<T, 4>& a);
    GLSL_VEC_COMMON(3)
};

template <class T> struct tvec<T, 4> {
    union {
        T v[4];
        struct { T x, y, z, w; };
        struct { T r, g, b, a; };
        swz<T, 4, 0, 1> xy;
        swz<T, 4, 2, 3> zw;
        swz<T, 4, 0, 1, 2> xyz;
        swz<T, 4, 0, 1, 2> rgb;
    };
    tvec() : v{T(0), T(0), T(0), T(0)} {}
    tvec(T a, T b, T c, T d) : v{a, b, c, d} {}
    explicit tvec(T s) : v{s, s, s, s} {}
    tvec(const tvec<T, 3>& a, T d) : v{a.v[0], a.v[1], a.v[2], d} {}
    tvec(const tvec<T, 2>& a, const tvec<T, 2>& b) : v{a.v[0], a.v[1], b.v[0], b.v[1]} {}
    GLSL_VEC_COMMON(4)
};
template <class T> inline tvec<T, 3>::tvec(const tvec<T, 4>& a) : v{a.v[0], a.v[1], a.v[2]} {}
#undef GLSL_VEC_COMMON

typedef tvec<float, 2> vec2;
typedef tvec<float, 3> vec3;
typedef tvec<float, 4> vec4;
typedef tvec<uint, 2> uvec2;
typedef tvec<uint, 3> uvec3;
typedef tvec<uint, 4> uvec4;
typedef tvec<int, 2> ivec2;
typedef tvec<int, 3> ivec3;
typedef tvec<int, 4> ivec4;
typedef tvec<bool, 2> bvec2;
typedef tvec<bool, 3> bvec3;
typedef tvec<bool, 4> bvec4;
static_assert(sizeof(vec3) == 12 && sizeof(vec4) == 16 && sizeof(uvec4) == 16 && sizeof(vec2) == 8, "std430 sizes");

struct mat4 { vec4 c[4]; };

/* Component-wise operators. The vector operand is a concrete type, so swizzle
 * views convert to it; scalars convert as GLSL allows. */
#define GLSL_BINOP(V, T, N, OP)                                                                              \
    inline V operator OP(const V& a, const V& b) { V r; for (int i = 0; i < N; ++i) r.v[i] = a.v[i] OP b.v[i]; return r; } \
    template <class S, class = std::enable_if_t<is_num_v<S> && (std::is_floating_point_v<T> || std::is_integral_v<S>)>> \
    inline V operator OP(const V& a, S s) { V r; for (int i = 0; i < N; ++i) r.v[i] = a.v[i] OP T(s); return r; } \
    template <class S, class = std::enable_if_t<is_num_v<S> && (std::is_floating_point_v<T> || std::is_integral_v<S>)>> \
    inline V operator OP(S s, const V& a) { V r; for (int i = 0; i < N; ++i) r.v[i] = T(s) OP a.v[i]; return r; } \
    inline V& operator OP##=(V& a, const V& b) { for (int i = 0; i < N; ++i) a.v[i] = a.v[i] OP b.v[i]; return a; } \
    template <class S, class = std::enable_if_t<is_num_v<S> && (std::is_floating_point_v<T> || std::is_integral_v<S>)>> \
    inline V& operator OP##=(V& a, S s) { for (int i = 0; i < N; ++i) a.v[i] = a.v[i] OP T(s); return a; }

#define GLSL_VEC_OPS(V, T, N)                                                                                \
    GLSL_BINOP(V, T, N, +) GLSL_BINOP(V, T, N, -) GLSL_BINOP(V, T, N, *) GLSL_BINOP(V, T, N, /)             \
    inline V operator-(const V& a) { V r; for (int i = 0; i < N; ++i) r.v[i] = -a.v[i]; return r; }        \
    inline bool operator==(const V& a, const V& b) { for (int i = 0; i < N; ++i) if (!(a.v[i] == b.v[i])) return false; return true; } \
    inline bool operator!=(const V& a, const V& b) { return !(a == b); }                                    \
    inline V min(const V& a, const V& b) { V r; for (int i = 0; i < N; ++i) r.v[i] = smin<T>(a.v[i], b.v[i]); return r; } \
    inline V max(const V& a, const V& b) { V r; for (int i = 0; i < N; ++i) r.v[i] = smax<T>(a.v[i], b.v[i]); return r; } \
    inline V min(const V& a, T b) { return min(a, V(b)); }                                                 \
    inline V max(const V& a, T b) { return max(a, V(b)); }                                                 \
    inline V clamp(const V& x, const V& lo, const V& hi) { return min(max(x, lo), hi); }                   \
    inline V clamp(const V& x, T lo, T hi) { return min(max(x, V(lo)), V(hi)); }

#define GLSL_INT_OPS(V, T, N)                                                                                \
    GLSL_BINOP(V, T, N, %) GLSL_BINOP(V, T, N, &) GLSL_BINOP(V, T, N, |) GLSL_BINOP(V, T, N, ^)             \
    GLSL_BINOP(V, T, N, <<) GLSL_BINOP(V, T, N, >>)

#define GLSL_FLOAT_FUNCS(V, N)                                                                               \
    inline float dot(const V& a, const V& b) { float s = a.v[0] * b.v[0]; for (int i = 1; i < N; ++i) s = s + a.v[i] * b.v[i]; return s; } \
    inline float length(const V& a) { return std::sqrt(dot(a, a)); }                                       \
    inline float distance(const V& a, const V& b) { return length(a - b); }                                \
    inline V normalize(const V& a) { return a / length(a); }                                               \
    inline V abs(const V& a) { V r; for (int i = 0; i < N; ++i) r.v[i] = std::fabs(a.v[i]); return r; }    \
    inline V floor(const V& a) { V r; for (int i = 0; i < N; ++i) r.v[i] = std::floor(a.v[i]); return r; } \
    inline V fract(const V& a) { V r; for (int i = 0; i < N; ++i) r.v[i] = fract(a.v[i]); return r; }      \
    inline V sqrt(const V& a) { V r; for (int i = 0; i < N; ++i) r.v[i] = std::sqrt(a.v[i]); return r; }   \
    inline V pow(const V& a, const V& b) { V r; for (int i = 0; i < N; ++i) r.v[i] = std::pow(a.v[i], b.v[i]); return r; } \
    inline V mix(const V& x, const V& y, float a) { return x * (1.0f - a) + y * a; }                       \
    inline V mix(const V& x, const V& y, const V& a) { return x * (V(1.0f) - a) + y * a; }                 \
    inline V mix(const V& x, const V& y, const tvec<bool, N>& s) { V r; for (int i = 0; i < N; ++i) r.v[i] = s.v[i] ? y.v[i] : x.v[i]; return r; } \
    inline V reflect(const V& i, const V& n) { return i - 2.0f * dot(n, i) * n; }                          \
    inline tvec<bool, N> lessThan(const V& a, const V& b) { tvec<bool, N> r; for (int i = 0; i < N; ++i) r.v[i] = a.v[i] < b.v[i]; return r; } \
    inline tvec<bool, N> greaterThan(const V& a, const V& b) { tvec<bool, N> r; for (int i = 0; i < N; ++i) r.v[i] = a.v[i] > b.v[i]; return r; }

GLSL_VEC_OPS(vec2, float, 2) GLSL_VEC_OPS(vec3, float, 3) GLSL_VEC_OPS(vec4, float, 4)
GLSL_VEC_OPS(uvec2, uint, 2) GLSL_VEC_OPS(uvec3, uint, 3) GLSL_VEC_OPS(uvec4, uint, 4)
GLSL_VEC_OPS(ivec2, int, 2) GLSL_VEC_OPS(ivec3, int, 3) GLSL_VEC_OPS(ivec4, int, 4)
GLSL_INT_OPS(uvec2, uint, 2) GLSL_INT_OPS(uvec3, uint, 3) GLSL_INT_OPS(uvec4, uint, 4)
GLSL_INT_OPS(ivec2, int, 2) GLSL_INT_OPS(ivec3, int, 3) GLSL_INT_OPS(ivec4, int, 4)
GLSL_FLOAT_FUNCS(vec2, 2) GLSL_FLOAT_FUNCS(vec3, 3) GLSL_FLOAT_FUNCS(vec4, 4)
#undef GLSL_BINOP
#undef GLSL_VEC_OPS
#undef GLSL_INT_OPS
#undef GLSL_FLOAT_FUNCS

inline vec3 cross(const vec3& a, const vec3& b) {
    return vec3(a.v[1] * b.v[2] - a.v[2] * b.v[1], a.v[2] * b.v[0] - a.v[0] * b.v[2], a.v[0] * b.v[1] - a.v[1] * b.v[0]);
}
template <int N> inline bool any(const tvec<bool, N>& b) { for (int i = 0; i < N; ++i) if (b.v[i]) return true; return false; }
template <int N> inline bool all(const tvec<bool, N>& b) { for (int i = 0; i < N; ++i) if (!b.v[i]) return false; return true; }

/* ---------------------------------------------------------------- invocation state */
inline uvec3 gl_GlobalInvocationID, gl_NumWorkGroups, gl_WorkGroupID, gl_LocalInvocationID;
inline uint gl_LocalInvocationIndex = 0;
/* Bit 0: a texture was sampled (the test scenes have no textures, so the bound
 * samplers are empty); bit 1: an image index was out of range. */
inline uint g_refglsl_error = 0;
inline void barrier() {}
inline void memoryBarrierShared() {}
inline uint atomicAdd(uint& m, uint v) { uint o = m; m += v; return o; }
template <class T> inline T nonuniformEXT(T x) { return x; }

/* ---------------------------------------------------------------- buffers and images */
template <class T> struct ssbo {
    T* p = nullptr;
    uint64_t n = 0;
    T scratch{};
    void bind(const void* ptr, uint64_t bytes) { p = (T*)ptr; n = ptr ? bytes / sizeof(T) : 0; }
    T& operator[](uint64_t i) {
        if (i < n) return p[i];
        scratch = T();
        return scratch;
    }
    uint length() const { return (uint)n; }
};

struct sampler2D { int unit = 0; };
inline vec4 texture(const sampler2D&, const vec2&) { g_refglsl_error |= 1u; return vec4(1.0f); }
inline vec4 textureLod(const sampler2D&, const vec2&, float) { g_refglsl_error |= 1u; return vec4(1.0f); }


/* rgba16f 3D image: four halves per texel, x fastest. */
struct image3D {
    uint16_t* data = nullptr;
    int w = 0, h = 0, d = 0;
    bool inside(const ivec3& c) const { return c.x >= 0 && c.y >= 0 && c.z >= 0 && c.x < w && c.y < h && c.z < d; }
    uint64_t at(const ivec3& c) const { return 4ull * (((uint64_t)c.z * h + c.y) * w + c.x); }
};
inline float half_to_float(uint16_t h) { _Float16 f; std::memcpy(&f, &h, 2); return (float)f; }
inline uint16_t float_to_half(float x) { _Float16 f = (_Float16)x; uint16_t h; std::memcpy(&h, &f, 2); return h; }
inline vec4 imageLoad(const image3D& im, const ivec3& c) {
    if (!im.inside(c)) { g_refglsl_error |= 2u; return vec4(0.0f); }
    const uint16_t* t = im.data + im.at(c);
    return vec4(half_to_float(t[0]), half_to_float(t[1]), half_to_float(t[2]), half_to_float(t[3]));
}
inline void imageStore(image3D& im, const ivec3& c, const vec4& v) {
    if (!im.inside(c)) { g_refglsl_error |= 2u; return; }
    uint16_t* t = im.data + im.at(c);
    for (int i = 0; i < 4; ++i) t[i] = float_to_half(v.v[i]);
}

/* rgba16f 2D image (x fastest); with no storage bound, stores are dropped. */
struct image2D {
    uint16_t* data = nullptr;
    int w = 0, h = 0;
};
inline void imageStore(image2D& im, const ivec2& c, const vec4& v) {
    if (!im.data) return;
    if (c.x < 0 || c.y < 0 || c.x >= im.w || c.y >= im.h) { g_refglsl_error |= 2u; return; }
    uint16_t* t = im.data + 4ull * ((uint64_t)c.y * im.w + c.x);
    for (int i = 0; i < 4; ++i) t[i] = float_to_half(v.v[i]);
}

}  // namespace glsl

#define GLSL_SSBO(T, name) static ::glsl::ssbo<T> name;
#define shared static
