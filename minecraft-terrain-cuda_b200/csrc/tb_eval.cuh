// Element-wise operators of density-function evaluation shared by the generated
// evaluators (volume and point paths). Semantics: cpu/include/mccuda/df_ops.h.
#pragma once

#include "tb_math.cuh"
#include "tb_noise.cuh"
#include "tb_rng.cuh"

namespace tb {

TB_HD TB_FI float cube_f(float x) { return x * x * x; }
TB_HD TB_FI float leaky(float x, float k) { return x > 0.0f ? x : x * k; }

// squeeze: c = clamp(x, -1, 1); c / 2 - c^3 / 24
TB_HD TB_FI float squeeze(float x) {
    const float c = jclamp(x, -1.0f, 1.0f);
    return c / 2.0f - cube_f(c) / 24.0f;
}

// GradientFunction with its tiling: 0 clamp to edge, 1 repeat, 2 mirrored repeat.
// factor = (to_value - from_value) / (to - from), computed in float at compile time.
TB_HD TB_FI float gradient_value(int mode, int32_t from, int32_t lo, int32_t hi, int32_t range, float from_value, float factor, int32_t c) {
    if (mode == 0) {
        const int32_t cl = c < lo ? lo : (c > hi ? hi : c);
        return from_value + static_cast<float>(cl - from) * factor;
    }
    const int32_t rel = iadd(c, -from);
    if (mode == 1) return from_value + static_cast<float>(fmod_i(rel, range)) * factor;
    const int32_t tile = fdiv(rel, range);
    const int32_t local = rel - tile * range;
    return (tile & 1) == 0 ? from_value + static_cast<float>(local) * factor : from_value + static_cast<float>(range - local) * factor;
}

}  // namespace tb
