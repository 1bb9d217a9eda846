// Shared device helpers of the ausaxs_b200 kernels (sm_100a).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace ausaxs_b200 {

constexpr int kNff = 15;        // settings::form_factor::max_ff_types (include/core/settings/FormFactorSettings.h:12)
constexpr int kExv = 0;         // form_factor::exv_bin   (include/core/form_factor/FormFactorType.h:33)
constexpr int kWater = 1;       // form_factor::water_bin (FormFactorType.h:34)
constexpr int kMaxTypes = 15;   // distinct atom form-factor types one structure may use
constexpr float kMagic = 12582912.0f;      // 1.5 * 2^23: x + kMagic rounds x to an integer, ties to even
constexpr int32_t kMagicBits = 0x4B400000; // bit pattern of kMagic
constexpr int kResBits = 16;              // bits of the fixed-point in-bin offset (see pair_residual)
constexpr int32_t kResBias = 1 << (kResBits - 1);  // bias making the offset non-negative
// inner points between drains of the 32-bit offset accumulators: TILE x segment <= 2^16 pairs per bin,
// each adding < 2^16, so a drained word stays below 2^32
template <int TILE>
__host__ __device__ constexpr int drain_segment() { return 65536 / TILE; }

// ---------------------------------------------------------------------------------------------
// Pair evaluation with the reference's rounding sequence.
// SIMD evaluators (include/core/hist/detail/data/CompactCoordinatesXYZW.h:382-423, :491-535,
// :602-655): d2 = (dx*dx + dy*dy) + dz*dz, d = sqrt(d2), bin = cvt_rn(d * inv_w); every operation
// rounded on its own (the squares are formed before lane shuffles, so nothing contracts), ties to
// even.  The scalar evaluator used for the last (len mod 4) partners of each row
// (CompactCoordinatesXYZW.h:303-307, IntrinsicHelpers.h:9-14) is contracted by the reference's
// release build (GCC -O3 -ffast-math -march=x86-64-v3) to fma(dz, dz, fma(dx, dx, dy*dy)) and
// rounds ties away from zero (std::round).
// ---------------------------------------------------------------------------------------------
struct PairBin {
    float d;    // distance (float, as the reference accumulates it)
    float xr;   // bin index as float
    int32_t bin;
};

__device__ __forceinline__ PairBin pair_eval(float4 a, float4 b, float inv_w, bool tail) {
    float dx = __fsub_rn(a.x, b.x);
    float dy = __fsub_rn(a.y, b.y);
    float dz = __fsub_rn(a.z, b.z);
    float s = __fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), __fmul_rn(dz, dz));
    if (tail) s = __fmaf_rn(dz, dz, __fmaf_rn(dx, dx, __fmul_rn(dy, dy)));
    PairBin r;
    r.d = __fsqrt_rn(s);
    float x = __fmul_rn(r.d, inv_w);
    float xm = __fadd_rn(x, kMagic);               // exact rint for 0 <= x < 2^22
    r.bin = __float_as_int(xm) - kMagicBits;
    r.xr = __fsub_rn(xm, kMagic);
    if (tail && __fsub_rn(x, r.xr) == 0.5f) {      // std::round: ties away from zero
        r.bin += 1;
        r.xr = __fadd_rn(r.xr, 1.0f);
    }
    // NaN / inf / huge distances: make the bin fail every range check
    if (!(x < 4194304.0f)) r.bin = 0x7fffffff;
    return r;
}

// pair_eval without the scalar-tail rule (the SIMD evaluators), with the range check folded into the
// magic-number rounding: xm = kMagic + rint(x) exactly while x < 2^22, so rint(x) < nbins is
// xm < kMagic + nbins (bin_limit, exact in float); NaN, infinite and huge distances fail it too.
__device__ __forceinline__ bool pair_eval_simd(float4 a, float4 b, float inv_w, float bin_limit, PairBin& r) {
    const float dx = __fsub_rn(a.x, b.x);
    const float dy = __fsub_rn(a.y, b.y);
    const float dz = __fsub_rn(a.z, b.z);
    const float s = __fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), __fmul_rn(dz, dz));
    r.d = __fsqrt_rn(s);
    const float xm = __fadd_rn(__fmul_rn(r.d, inv_w), kMagic);
    if (!(xm < bin_limit)) return false;
    r.bin = __float_as_int(xm) - kMagicBits;
    r.xr = __fsub_rn(xm, kMagic);
    return true;
}
__host__ __device__ inline float pair_bin_limit(int nbins) {
    return kMagic + static_cast<float>(nbins < (1 << 22) ? nbins : (1 << 22));
}

// Square root by one Newton-Raphson correction of the hardware reciprocal-square-root approximation
// (Markstein's formulation: d0 = s y, r = s - d0^2 exactly by an FMA, d = d0 + r y / 2).  It differs
// from the correctly rounded root by at most one unit in the last place on a small fraction of
// inputs; the pair kernel uses it only for bin widths at which an exhaustive device check
// (pair_sqrt_prepare) found that no float input lands in another bin under either rounding rule of
// the reference, so bins stay exact and the distance sums move by at most one ulp of a distance.
__device__ __forceinline__ float pair_sqrt_nr(float s) {
    float y;
    asm("rsqrt.approx.f32 %0, %1;" : "=f"(y) : "f"(fmaxf(s, 1.17549435e-38f)));  // finite at s = 0
    const float d0 = __fmul_rn(s, y);
    const float h = __fmul_rn(0.5f, y);
    return __fmaf_rn(__fmaf_rn(-d0, d0, s), h, d0);
}

// Fixed-point in-bin offset of a pair: the distance is d = bin*c + r with |r| <= c/2 (1 + 2^-10)
// (c = 1/inv_w rounded to float), r is stored as rint(r * scale) + kResBias in [0, 2^16) with
// scale = 2^15 / c * (1 - 2^-8).  Sums of these are exact integers, so the per-bin mean distance
// does not depend on summation order; the quantisation step is about c * 2^-15 (7.6e-6 A at the
// default 0.25 A bins, 3.1e-6 A at 0.1 A), and rounding errors of many pairs average out.
__device__ __forceinline__ uint32_t pair_residual(const PairBin& p, float c, float scale) {
    float r = __fmaf_rn(-p.xr, c, p.d);
    float t = __fmaf_rn(r, scale, kMagic);  // rint(r * scale), one rounding
    return static_cast<uint32_t>(__float_as_int(t) - kMagicBits + kResBias);
}


// ---------------------------------------------------------------------------------------------
// Five-Gaussian atomic form factors f(q) = sum_i a_i exp(-b_i q^2) + c, with b tabulated in
// s = q / (4 pi) units (converted by 1 / (16 pi^2)), indexed by form_factor_t
// (include/core/form_factor/FormFactorTable.h:8-186, FormFactor.h:33-39).
// Published coefficients: Waasmaier & Kirfel, Acta Cryst. A51 (1995) for C, N, O, S and Ar
// (OTHER); International Tables for H; Grudinin, Garkavenko & Kazennov, Acta Cryst. D73 (2017)
// for the united-atom groups.  Entry 0 is the reference's average excluded-volume form factor
// a = {1}, b = {r^2/2} with r = 1.62 A, not converted (FormFactorTable.h, excluded_volume).
// ---------------------------------------------------------------------------------------------
struct FormFactor5 {
    double a[5], b[5], c;
};

}  // namespace ausaxs_b200
