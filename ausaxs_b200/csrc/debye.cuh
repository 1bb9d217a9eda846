// Debye transform of the compact histograms (see debye.cu, debye_tc.cu).
#pragma once
#include "common.cuh"

namespace ausaxs_b200 {

// What a histogram row contributes to, and with which form-factor product.
enum RowKind : int32_t {
    kRowAA = 0,   // F(ta, tb)                                    -> aa
    kRowAX = 1,   // 2 crho cx F(ta, exv)                          -> ax
    kRowXX = 2,   // (cx crho)^2 F(exv, exv)                       -> xx
    kRowAW = 3,   // 2 cw F(ta, water)                             -> aw
    kRowWX = 4,   // 2 crho cx cw F(exv, water)                    -> wx
    kRowWW = 5,   // cw^2 F(water, water)                          -> ww
    kRowSAA = 6,  // Simple: exp(-q^2)                             -> aa
    kRowSAW = 7,  // Simple: exp(-q^2) (I gets cw)                 -> aw
    kRowSWW = 8   // Simple: exp(-q^2) (I gets cw^2)               -> ww
};

struct RowDesc {
    int32_t group;  // which distance axis: 0 = aa, 1 = ax/wx, 2 = xx
    int32_t kind;   // RowKind
    int32_t ta, tb; // form_factor_t of the two sides (atoms)
};

struct DebyeArgs {
    int32_t R;
    int32_t nb;                 // row stride
    const double* H;            // [R][nb]
    const double* axis0;        // d-axis of group 0
    const double* axis1;        // group 1 (may equal axis0)
    const double* axis2;        // group 2
    const int32_t* max_bin;     // device int: bins in use
    const RowDesc* rows;        // [R]
    const unsigned long long* overflow;  // non-zero: the histogram lost pairs, I(q) is set to NaN
    int32_t exv_model;          // 0: average exv form factor (FFAvg), 1: grid dummies of volume V
    double cw, cx, crho, dw_atomic, dw_exv, grid_volume;
    const double* q;
    int32_t nq;
    const float* sinqd_tc;      // [R][nq] from the tensor-core contraction, or null (FP64 everywhere)
    const float* bound_tc;      // [R][nq] sum_b |H| |sinc| estimate, or null
    double tolerance;           // relative I(q) error target when sinqd_tc is given
    int32_t* fp64_columns;      // out: number of q recomputed in FP64 (may be null)
    double* Iq;                 // [nq]
    double* profiles;           // [6][nq] or null
};

void debye_fp64_launch(const DebyeArgs& A, cudaStream_t s);

// Split-BF16 tensor-core contraction sinqd[r][q] = sum_b H[r][b] sinc(q d_{g(r)}[b]) for all rows,
// with a bound sum_b |H||sinc| per element; returns false when the launch could not be made
// (then callers use the FP64 path).
struct TcArgs {
    int32_t R, nb;
    const double* H;
    const double* axis0;
    const double* axis1;
    const double* axis2;
    const RowDesc* rows;
    const int32_t* max_bin;
    const double* q;
    int32_t nq;
    float* sinqd;  // [R][nq]
    float* bound;  // [R][nq]
    // scratch
    unsigned short* a_hi;  // [Mpad][Kpad] bf16 packed in UMMA layout
    unsigned short* a_lo;
    int32_t kpad, mpad;
};
bool debye_tc_launch(const TcArgs& A, int bins_hint, cudaStream_t s);
size_t debye_tc_scratch_bytes(int R, int bins_hint);

}  // namespace ausaxs_b200
