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
    kRowSWW = 8,  // Simple: exp(-q^2) (I gets cw^2)               -> ww
    // FFExplicit (CompositeDistanceHistogramFFExplicitBase.cpp:64-211): one aa row serves three
    // profiles, one aw row two, with per-type excluded-volume form factors x_t and e(q)
    kRowEAA = 9,  // F(ta,tb) -> aa;  crho e (f_ta x_tb + f_tb x_ta) -> ax;  (e crho)^2 x_ta x_tb -> xx
    kRowEAW = 10, // 2 cw F(ta,w) -> aw;  crho e cw (f_w x_ta + f_ta x_w) -> wx
    kRowZero = 11 // not used by this transform (FFExplicit's exv marginal rows)
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
    int32_t exv_model;          // 0: average exv form factor (FFAvg), 1: grid dummies of volume V,
                                // 2: per-type excluded volumes (FFExplicit)
    double cw, cx, crho, dw_atomic, dw_exv, grid_volume;
    const double* q;
    int32_t nq;
    // tensor-core partial sums from debye_tc_launch, or null (FP64 for every q):
    //   sinqd_tc [splits][R][nq], bound_tc [splits][R][nq] (sum_b |H| |sinc|), habs_tc [splits][R] (sum_b |H|)
    const float* sinqd_tc;
    const float* bound_tc;
    const float* habs_tc;
    int32_t tc_splits;          // K splits of the bin range
    const int32_t* tc_error;    // non-zero: the tensor-core values are unusable (FP64 for every q)
    double tolerance;           // relative I(q) error target when sinqd_tc is given
    int32_t* fp64_columns;      // out: number of q recomputed in FP64 (may be null)
    double* tc_err_est;         // out: [nq] estimated relative error of the tensor-core I(q) (may be null)
    double* Iq;                 // [nq]
    double* profiles;           // [6][nq] or null
    // exact-accumulation tensor-core partial sums from debye_x_enqueue, or null (debye_x.cu):
    //   x_v [x_splits][R][nq] (FP64 values), x_e1 / x_e0 / x_habs [x_splits][R] (bound terms: the error of
    //   a split's value is at most x_e1 * Csum(q) + x_e0, Csum(q) = sum_c x_cpart[c][q] over x_nch
    //   table chunks), and the Taylor truncation x_ctr * q^x_K * sum_z x_habs
    const double* x_v;
    const double* x_e1;
    const double* x_e0;
    const double* x_habs;
    int32_t x_splits;
    const double* x_cpart;      // [x_nch][x_nqp]
    int32_t x_nch, x_nqp, x_K;
    double x_ctr;
    // per-q factors made by debye_qfactors_launch for transforms sharing q, the parameters and the
    // excluded-volume model, or null (each CTA evaluates its own)
    const double* qf;
};

void debye_fp64_launch(const DebyeArgs& A, cudaStream_t s);
// The per-q factor table (form factors, excluded-volume and Debye-Waller factors) of A's q values and
// parameters into out [debye_qfactors_doubles(nq)]
size_t debye_qfactors_doubles(int nq);
void debye_qfactors_launch(const DebyeArgs& A, double* out, cudaStream_t s);
// n transforms at once (device array of arguments; max_nq >= every nq, max_R >= every R)
void debye_fp64_batch_launch(const DebyeArgs* As_dev, int n, int max_nq, int max_R, cudaStream_t s);

// Split-BF16 tensor-core contraction sinqd[r][q] = sum_b H[r][b] sinc(q d_{g(r)}[b]) for all rows,
// with the bound sum_b |H||sinc| per element (debye_tc.cu).  Returns false when the launch could not
// be made (callers then use FP64 for every q).
struct TcArgs {
    int32_t R, nb, nq;
    const double* H;
    const double* axis0;
    const double* axis1;
    const double* axis2;
    const RowDesc* rows;
    const int32_t* max_bin;
    const double* q;
    int32_t groups_present;  // bit g: some row uses distance axis g
    int32_t splits;          // K splits of the bin range (tc_splits)
    float* sinqd;            // [splits][R][nq]
    float* bound;            // [splits][R][nq]
    float* habs;             // [splits][R]
    int32_t* error_flag;
};
bool debye_tc_launch(const TcArgs& A, cudaStream_t s);
// K splits for a contraction of up to `bins` bins, R rows, nq q values and `groups` distance axes
// (fills the SMs once)
int debye_tc_splits(int R, int bins, int nq, int sms, int groups);
// bins of one K split when max_bin bins are in use (multiple of the 64-bin staging chunk)
__host__ __device__ inline int debye_tc_split_bins(int max_bin, int splits) {
    const int chunks = (max_bin + 63) / 64;
    return ((chunks + splits - 1) / splits) * 64;
}
size_t debye_tc_smem_bytes();

// Exact-accumulation tensor-core contraction over shared Taylor tables (debye_x.cu).
// One left-operand row: a histogram row of some structure and where its partial sums go.
struct XRow {
    const double* H;         // the row's bins (null: a padding row)
    const double* axis;      // its distance axis
    const int32_t* max_bin;  // its structure's bins in use (device)
    double* out;             // value of split z, q value k: out[z * out_z + k]
    double* e1;              // bound terms of split z: e1[z * e_z], e0[z * e_z], habs[z * e_z]
    double* e0;
    double* habs;
    long long out_z;
    int32_t e_z;
    int32_t pad;
};
constexpr int kXChunk = 64;     // bins per table chunk
constexpr int kXQTile = 64;     // q values per table tile
constexpr int kXMaxOrder = 8;   // Taylor orders at most
// Taylor orders for q values up to qmax at bin width w: the truncation (qmax w / 2)^K / (K! (K + 1))
// below 2^-32 of sum |H| (at least 2, at most kXMaxOrder)
int debye_x_order(double qmax, double w);
// (w / 2)^K 1.01^K / (K! (K + 1)): times q^K sum |H|, the truncation bound (|u| <= 1.01)
double debye_x_trunc(int K, double w);
// chunks one split may hold for K orders (its s32 sums stay exact)
int debye_x_max_chunks(int K);
size_t debye_x_table_bytes(int nq, int nch, int K);
size_t debye_x_cpart_doubles(int nq, int nch);
// bytes of the rows' digit block of one (M tile, chunk, order)
size_t debye_x_block_bytes();
// Device buffers and shape of one contraction (rows in M tiles of 128 consecutive rows).
struct XPlan {
    const XRow* rows;
    int n_rows, nq, nch, K, cps, splits;
    double w;
    unsigned char* table;      // debye_x_table_bytes(nq, nch, K)
    double* cpart;             // debye_x_cpart_doubles(nq, nch): per chunk and q, sum_{k, b} |C_k(b, q)|
    double* q_cached;          // [nq]: the q the tables were made for (NaN: none yet)
    int32_t* flags;            // [0] tables stale, [1] error (sticky: every later transform in FP64)
    unsigned char* adig;       // the rows' digit blocks: tile t, chunk c, order k at tile_off[t] + (c K + k) block
    const long long* tile_off;  // [M tiles]
    double* row_scale;         // [n_rows]
};
// q check and tables (rebuilt only when q changed), row scales and bound terms, the rows' digits and
// the contraction, on stream s; false when a launch could not be made
bool debye_x_enqueue(const XPlan& X, const double* q, cudaStream_t s);

}  // namespace ausaxs_b200
