// probe_dirs.cpp -- ray directions and SH9 basis weights for light-probe updates
// (include/tim_rt.h, tim_rt_probe_directions), host only.
//   stratified: LightProbFieldPass::sampleRays (src/Renderer/lightProbFieldPass.cpp:151-202):
//     cell (i, j) of a side x side grid, r = ((i, j) + U^2) / side, theta = 2 pi r.x,
//     phi = acos(1 - 2 r.y), N = (sin phi cos theta, sin phi sin theta, cos phi), ray
//     index i * side + j, drawn with std::uniform_real_distribution<float> from a
//     std::mt19937 seeded by the caller (the reference draws from std::random_device,
//     so its directions are not reproducible);
//   octahedral: the centres of a side x side octahedral grid, index j * side + i (the
//     layout TIM_RT_PROBE_OCTA bins into 8 x 8 texels).
// SH9 weights: the constants and order of sampleRays (lightProbFieldPass.cpp:186-199).
#include <cmath>
#include <random>
#include "tim_rt.h"
#include "internal.h"

using timrt::set_error;

namespace {

constexpr float kPi = 3.14159265358979323846f;   // TIM_PI, timCore/type.h:5

void sh9(float x, float y, float z, float* w) {
    w[0] = 0.282095f;                        // SH_Y00
    w[1] = 0.488603f * x;                    // SH_Y11
    w[2] = 0.488603f * z;                    // SH_Y10
    w[3] = 0.488603f * y;                    // SH_Y1_1
    w[4] = 1.092548f * x * z;                // SH_Y21
    w[5] = 1.092548f * y * z;                // SH_Y2_1
    w[6] = 1.092548f * x * y;                // SH_Y2_2
    w[7] = 0.315392f * (3.0f * z * z - 1.0f);  // SH_Y20
    w[8] = 0.546274f * (x * x - y * y);      // SH_Y22
}

}  // namespace

extern "C" int tim_rt_probe_directions(uint32_t count, uint32_t kind, uint64_t seed, float* dirs, float* sh_basis) {
    uint32_t side = 0;
    while (side * side < count) ++side;
    if (!dirs || count == 0 || count > 4096 || side * side != count ||
        (kind != TIM_RT_DIRS_STRATIFIED && kind != TIM_RT_DIRS_OCTAHEDRAL)) {
        set_error("tim_rt_probe_directions: count must be a square of 1..4096, kind STRATIFIED or OCTAHEDRAL");
        return TIM_RT_EINVAL;
    }
    if (kind == TIM_RT_DIRS_STRATIFIED) {
        std::mt19937 rng((std::mt19937::result_type)(seed ^ (seed >> 32)));
        std::uniform_real_distribution<float> uniform01(0, 1);
        for (uint32_t i = 0; i < side; ++i)
            for (uint32_t j = 0; j < side; ++j) {
                const float cx = float(i) / side, cy = float(j) / side;
                float rx = uniform01(rng), ry = uniform01(rng);
                rx = rx / side;
                ry = ry / side;
                rx = rx + cx;
                ry = ry + cy;
                const float theta = 2 * kPi * rx;
                const float phi = std::acos(1 - 2 * ry);
                const float x = std::sin(phi) * std::cos(theta);
                const float y = std::sin(phi) * std::sin(theta);
                const float z = std::cos(phi);
                const uint32_t k = i * side + j;
                dirs[4 * k] = x; dirs[4 * k + 1] = y; dirs[4 * k + 2] = z; dirs[4 * k + 3] = 0.f;
                if (sh_basis) sh9(x, y, z, sh_basis + 9 * k);
            }
    } else {
        for (uint32_t j = 0; j < side; ++j)
            for (uint32_t i = 0; i < side; ++i) {
                double x = (i + 0.5) / side * 2.0 - 1.0, y = (j + 0.5) / side * 2.0 - 1.0;
                const double z = 1.0 - std::fabs(x) - std::fabs(y);
                if (z < 0) {   // fold the lower hemisphere
                    const double xo = x, yo = y;
                    x = (1.0 - std::fabs(yo)) * (xo < 0 ? -1.0 : (xo > 0 ? 1.0 : 0.0));
                    y = (1.0 - std::fabs(xo)) * (yo < 0 ? -1.0 : (yo > 0 ? 1.0 : 0.0));
                }
                const double len = std::sqrt(x * x + y * y + z * z);
                const uint32_t k = j * side + i;
                dirs[4 * k] = (float)(x / len); dirs[4 * k + 1] = (float)(y / len); dirs[4 * k + 2] = (float)(z / len);
                dirs[4 * k + 3] = 0.f;
                if (sh_basis) sh9(dirs[4 * k], dirs[4 * k + 1], dirs[4 * k + 2], sh_basis + 9 * k);
            }
    }
    return TIM_RT_OK;
}
