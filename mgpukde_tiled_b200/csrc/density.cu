// Density gather over the cell-binned index (one raster tile per call).
//
// Reference: KernelDesityEstimation_pPoints (kde_kernel_kdtr.cu:461-574) scatters
// each point's window into the tile with float atomicAdd, after
// InitCellDensities (:268-294) zeroed the valid cells.  Here every cell is
// owned by one thread that gathers:
//
//   den(c) = sum_p [d^2 < 9 h_p^2] exp(-d^2 / 2 h_p^2) / (h_p^2 TWO_PI) w_p e_p
//
// Layout: a CTA (256 threads) owns a 64 x 128 block of cells; warp w owns a
// 32 x 32 sub-block, lane l a 4 x 8 micro-tile.  A block whose cells are all
// NoData stages no candidates and writes NoData (the reference skips NoData
// cells, kde_kernel_kdtr.cu:426-428).  Candidates (points of the bins within
// 3h of the block, one contiguous range per bin row) arrive in mini-batches
// of 64, taken by two cursors across bin rows, through a double-buffered TMA
// bulk copy (cp.async.bulk + mbarrier) into shared memory; the next batch is
// staged during the current batch's phase B by the warp with the fewest
// points to sum.  Per mini-batch:
//
//  phase A (all 256 threads, 8 per point): each warp's sub-block first gets
//    an exact-enough rectangle-vs-disc test (skip, fully inside, partial).
//    The Gaussian factorises over the grid, exp2(-(a_j + b_i)) = E_j F_i with
//    a_j = dx_j^2 k2, b_i = dy_i^2 k2, k2 = log2(e) / (2 h^2); the column
//    factors and row factors are built only for the column halves and warp
//    rows of the sub-blocks that sum the point.  Coordinates are hi/lo float
//    pairs on a common quantum, so dx = (xh - cxh) + (xl - cxl) is exact as a
//    pair and a = dx^2 k2 is formed with error-free float products (no FP64,
//    no conversions); E = ex2(-a_hi) (1 - a_lo ln2).  Row entries also carry
//    the cutoff threshold G_i = 2^-cut / 2^-b_i (a_j < cut - b_i <=>
//    E_j > G_i) and a flag marking rows where some column lies within a 4e-6
//    (log2 units) band of the cutoff.
//  phase B (each warp, its processed points): per cell one FFMA (fully
//    inside) or one compare E_j > G_i and a predicated FFMA part += E_j F_i.
//    Rows flagged as ambiguous are re-decided with the exact FP64 test of the
//    oracle, so the summed pair set is exactly the reference's.
//
// Accumulation: FP32 partial sums over 32 points per cell (registers), added
// into a Kahan-compensated FP32 accumulator in tensor memory (tcgen05: 128
// columns per CTA, sum and compensation of each thread's 32 cells in 64
// columns of its warp's lane quarter); the epilogue forms (s - c) times the
// kernel normalisation in FP64.  With 126-128 registers per thread two CTAs
// run per SM.  Heavy blocks are split into work items whose FP64 partials
// are merged in a fixed order, so results are bitwise reproducible.
#include <algorithm>
#include <cstring>
#include <cmath>
#include <mutex>
#include <vector>

#include "mgk_internal.cuh"

namespace {

constexpr int kThreads = 256;
constexpr int kBR = 64;         // cell rows of a CTA block
constexpr int kBC = 128;        // cell columns of a CTA block
constexpr int kCells = kBR * kBC;
constexpr int kMergeParts = 8;  // CTAs per split block in the merge kernels (kCells / 8 cells each)
constexpr int kMB = 64;         // points per mini-batch (a multiple of 32)
constexpr int kStage64 = 512;   // points staged per batch by the FP64 form
constexpr float kAmbEps = 4e-6f;
constexpr long long kSpinLimit = 1ll << 24;

struct Item {
    int32_t bx, by;       // block coordinates within the tile
    int32_t k0, k1;       // candidate range in the block's candidate sequence
    int32_t slot;         // scratch slot (split blocks) or -1 (direct store)
    int32_t pad;
};

struct DParams {
    double xll, yll, cs;
    int64_t g_nrows;
    int64_t row0, col0, nr, nc;
    float nodata;
    const float* mask;
    // the same NoData mask as bits (1 = valid; row r of the tile at byte
    // r * mbstride, column c at bit c % 8 of byte c / 8), used instead of
    // `mask` when set
    const unsigned char* mbits;
    int64_t mbstride;
    float* out;
    double* scratch;  // [slot][kCells]
    const Item* items;
    // index
    const MgkPt* pts;
    const int32_t* bin_start;
    double ox, oy, side, inv_side;
    int64_t nbx, nby;
    int qexp;
    // fixed-h constants
    double h2, k0, cut_d2, reach;
    float k2h, k2l, cutf, epsd2;
    float gcut;  // 2^-(cutoff in log2 units): the in-cutoff threshold on E_j F'_i
    unsigned long long* evals;
    unsigned long long* err;
    unsigned* tail_flag;  // set to 1 when the launch's last CTA starts (null: none)
};

// Is cell (rr, cc) of the tile (tile-relative) valid: inside the mask and not NoData?
__device__ __forceinline__ bool cell_valid(const DParams& P, int64_t rr, int64_t cc) {
    if (P.mbits) return (P.mbits[rr * P.mbstride + (cc >> 3)] >> (cc & 7)) & 1u;
    return !P.mask || P.mask[rr * P.nc + cc] != P.nodata;
}

// Bin range covering [lo, hi] (coordinates), clamped; returns false if empty.
__device__ __forceinline__ bool bin_range(double lo, double hi, double o, double inv_side, int64_t nb,
                                          int64_t& a, int64_t& b) {
    double fa = floor((lo - o) * inv_side), fb = floor((hi - o) * inv_side);
    if (fb < 0.0 || fa > (double)(nb - 1)) return false;
    a = fa < 0.0 ? 0 : (int64_t)fa;
    b = fb > (double)(nb - 1) ? nb - 1 : (int64_t)fb;
    return true;
}

struct BlockGeom {
    int64_t r0, c0;   // global first row / col of the block
    int nrow, ncol;   // cells of the block inside the tile
    int64_t bx0, bx1, by0, by1;
    double x_lo, x_hi, y_lo, y_hi;  // extent of the block's cell centres
    bool any;
};

__device__ __forceinline__ BlockGeom block_geom(const DParams& P, int bxi, int byi) {
    BlockGeom G;
    G.r0 = P.row0 + (int64_t)byi * kBR;
    G.c0 = P.col0 + (int64_t)bxi * kBC;
    G.nrow = (int)mgk_min64(kBR, P.row0 + P.nr - G.r0);
    G.ncol = (int)mgk_min64(kBC, P.col0 + P.nc - G.c0);
    G.x_lo = mgk_cell_x(P.xll, P.cs, G.c0);
    G.x_hi = mgk_cell_x(P.xll, P.cs, G.c0 + G.ncol - 1);
    G.y_hi = mgk_cell_y(P.yll, P.cs, P.g_nrows, G.r0);
    G.y_lo = mgk_cell_y(P.yll, P.cs, P.g_nrows, G.r0 + G.nrow - 1);
    G.any = bin_range(G.x_lo - P.reach, G.x_hi + P.reach, P.ox, P.inv_side, P.nbx, G.bx0, G.bx1) &&
            bin_range(G.y_lo - P.reach, G.y_hi + P.reach, P.oy, P.inv_side, P.nby, G.by0, G.by1);
    return G;
}

// Candidates of bin row `by` for the block: a point of the row can be within
// reach of a cell centre only if |x - [x_lo, x_hi]| <= sqrt(reach^2 - dy^2),
// dy the distance from the row's y-extent to [y_lo, y_hi] (a lower bound on
// the point's), so the row's bin range narrows away from the block (the
// candidate region is the block rectangle grown by a disc, not by a square).
// Returns the row's contiguous range [sb, sb + len) of the index.
__device__ __forceinline__ void row_span(const DParams& P, const BlockGeom& G, int64_t by, int64_t& sb,
                                         int64_t& len) {
    const double rlo = P.oy + (double)by * P.side, rhi = rlo + P.side;
    const double dy = fmax(0.0, fmax(rlo - G.y_hi, G.y_lo - rhi)) * (1.0 - 1e-9);
    const double rr = P.reach * P.reach - dy * dy;
    int64_t b0, b1;
    if (rr >= 0.0) {
        const double hw = sqrt(rr) * (1.0 + 1e-9) + 1e-9 * P.reach;
        if (bin_range(G.x_lo - hw, G.x_hi + hw, P.ox, P.inv_side, P.nbx, b0, b1)) {
            sb = P.bin_start[by * P.nbx + b0];
            len = (int64_t)P.bin_start[by * P.nbx + b1 + 1] - sb;
            return;
        }
    }
    sb = 0;
    len = 0;
}

// Candidate count of every block of the tile (planning).
__global__ void k_block_counts(DParams P, int nbx_t, int nby_t, int64_t* __restrict__ counts) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i == 0 && P.err) *P.err = 0;  // the staging-wait flag of the launch this plan is for
    if (i >= nbx_t * nby_t) return;
    const BlockGeom G = block_geom(P, i % nbx_t, i / nbx_t);
    int64_t c = 0;
    if (G.any)
        for (int64_t by = G.by0; by <= G.by1; by++) {
            int64_t sb, len;
            row_span(P, G, by, sb, len);
            c += len;
        }
    counts[i] = c;
}

__device__ __forceinline__ void kahan_add(float& s, float& c, float v) {
    const float y = v - c;
    const float t = s + y;
    c = (t - s) - y;
    s = t;
}

// kahan_add on two cells at once, in packed FP32 (add/sub.rn.f32x2): each
// half is bitwise the scalar form.
__device__ __forceinline__ void kahan_add2(float& s0, float& s1, float& c0, float& c1, float v0, float v1) {
    asm("{\n .reg .b64 s, c, v, y, t;\n mov.b64 s, {%0, %1};\n mov.b64 c, {%2, %3};\n mov.b64 v, {%4, %5};\n"
        " sub.rn.f32x2 y, v, c;\n add.rn.f32x2 t, s, y;\n sub.rn.f32x2 c, t, s;\n sub.rn.f32x2 c, c, y;\n"
        " mov.b64 {%0, %1}, t;\n mov.b64 {%2, %3}, c;\n}\n"
        : "+f"(s0), "+f"(s1), "+f"(c0), "+f"(c1)
        : "f"(v0), "f"(v1));
}

// ---- TMA bulk copy + mbarrier (sm_90+ PTX) ---------------------------------
__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* b, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(b)), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ void mbar_arrive_tx(uint64_t* b, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(b)), "r"(bytes) : "memory");
}
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, unsigned bytes, uint64_t* b) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(b))
                 : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* b, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(b)), "r"(parity)
        : "memory");
    return ok != 0;
}
// Bounded wait on an mbarrier phase; false when the limit ran out.
__device__ __forceinline__ bool mbar_wait(uint64_t* b, unsigned parity) {
    for (long long i = 0; i < kSpinLimit; i++)
        if (mbar_try_wait(b, parity)) return true;
    return false;
}

// ---- tensor memory (sm_100a tcgen05) ---------------------------------------
// The per-cell Kahan accumulators of a block live in tensor memory.  A warp
// may address only its quarter of the 128 TMEM lanes (warp w: lanes
// 32 (w % 4) ..); with the 32x32b shape thread t of the warp reads and writes
// lane 32 (w % 4) + t, one 32-bit column per register.  TMEM addresses carry
// the lane in bits 31:16 and the column in bits 15:0.
constexpr unsigned kTmemCols = 128;  // warps w and w + 4 share lanes: columns 64 (w / 4) .. + 64

__device__ __forceinline__ void tmem_alloc(unsigned* dst) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(dst)),
                 "r"(kTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(unsigned taddr) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(kTmemCols) : "memory");
}
__device__ __forceinline__ void tmem_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tmem_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tmem_wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }

// Columns taddr .. taddr + 7 of the thread's lane into v (valid on return:
// the wait names the registers, so no use of them moves above it).
__device__ __forceinline__ void tmem_ld8(unsigned taddr, float (&v)[8]) {
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                 : "=f"(v[0]), "=f"(v[1]), "=f"(v[2]), "=f"(v[3]), "=f"(v[4]), "=f"(v[5]), "=f"(v[6]), "=f"(v[7])
                 : "r"(taddr)
                 : "memory");
}
__device__ __forceinline__ void tmem_wait_ld(float (&a)[8], float (&b)[8]) {
    asm volatile("tcgen05.wait::ld.sync.aligned;"
                 : "+f"(a[0]), "+f"(a[1]), "+f"(a[2]), "+f"(a[3]), "+f"(a[4]), "+f"(a[5]), "+f"(a[6]), "+f"(a[7]),
                   "+f"(b[0]), "+f"(b[1]), "+f"(b[2]), "+f"(b[3]), "+f"(b[4]), "+f"(b[5]), "+f"(b[6]), "+f"(b[7])
                 :
                 : "memory");
}
__device__ __forceinline__ void tmem_st8(unsigned taddr, const float (&v)[8]) {
    asm volatile("tcgen05.st.sync.aligned.32x32b.x8.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8};" ::"r"(taddr),
                 "f"(v[0]), "f"(v[1]), "f"(v[2]), "f"(v[3]), "f"(v[4]), "f"(v[5]), "f"(v[6]), "f"(v[7])
                 : "memory");
}

// Exponent a = (t + lo)^2 (k2h + k2l) as a float pair ah + al.  t is exact
// (difference of two multiples of the quantum), |lo| <= quantum.  dx = t + lo
// is formed as an exact pair (dh, de) first, so p = dh^2 is the rounded
// square, pe its error-free remainder plus 2 dh de, and the products with k2
// are error-free: ah is a to within a few ulps (|al| <= ~3 ulp(ah)), and
// ah + al is a to about 2^-40 relative.  d2 = p + pe approximates dx^2.
__device__ __forceinline__ void exponent_pair(float t, float lo, float k2h, float k2l, float& ah, float& al,
                                              float& d2) {
    const float dh = __fadd_rn(t, lo);
    const float de = __fsub_rn(lo, __fsub_rn(dh, t));
    const float p = __fmul_rn(dh, dh);
    const float pe = __fmaf_rn(__fadd_rn(dh, dh), de, __fmaf_rn(dh, dh, -p));
    d2 = __fadd_rn(p, pe);
    ah = __fmul_rn(p, k2h);
    const float ae = __fmaf_rn(p, k2h, -ah);
    al = __fmaf_rn(pe, k2h, __fmaf_rn(p, k2l, ae));
}

// exponent_pair and exp2_pair of two entries at once, in packed FP32
// (f32x2).  The negations are arranged so that every half is bitwise the
// scalar form: fma(-a, b, c) = -fma(a, b, -c) under round-to-nearest, so pen
// = -pe and ahn = -ah exactly.  Returns the two factors 2^-(a_0), 2^-(a_1)
// and the approximate squares d2.
__device__ __forceinline__ void exp2_pair2(float t0, float t1, float lo0, float lo1, float k2h, float k2l,
                                           float& e0, float& e1, float& d20, float& d21) {
    float ahn0, ahn1, al0, al1;
    asm("{\n .reg .b64 t, lo, dh, tmp, de, p, dhn, err, dh2n, pen, kh, khn, kl, ahn, ae, x, al, d2;\n"
        " mov.b64 t, {%6, %7};\n mov.b64 lo, {%8, %9};\n"
        " mov.b64 kh, {%10, %10};\n mov.b64 kl, {%11, %11};\n mov.b64 khn, {%12, %12};\n"
        " add.rn.f32x2 dh, t, lo;\n sub.rn.f32x2 tmp, dh, t;\n sub.rn.f32x2 de, lo, tmp;\n"
        " mul.rn.f32x2 p, dh, dh;\n mov.b64 dhn, 0xBF800000BF800000;\n mul.rn.f32x2 dhn, dh, dhn;\n"
        " fma.rn.f32x2 err, dhn, dh, p;\n add.rn.f32x2 dh2n, dhn, dhn;\n fma.rn.f32x2 pen, dh2n, de, err;\n"
        " sub.rn.f32x2 d2, p, pen;\n mul.rn.f32x2 ahn, p, khn;\n fma.rn.f32x2 ae, p, kh, ahn;\n"
        " fma.rn.f32x2 x, p, kl, ae;\n fma.rn.f32x2 al, pen, khn, x;\n"
        " mov.b64 {%0, %1}, ahn;\n mov.b64 {%2, %3}, al;\n mov.b64 {%4, %5}, d2;\n}\n"
        : "=f"(ahn0), "=f"(ahn1), "=f"(al0), "=f"(al1), "=f"(d20), "=f"(d21)
        : "f"(t0), "f"(t1), "f"(lo0), "f"(lo1), "f"(k2h), "f"(k2l), "f"(-k2h));
    const float x0 = mgk_ex2(ahn0), x1 = mgk_ex2(ahn1);
    asm("{\n .reg .b64 al, c, x, e;\n mov.b64 al, {%2, %3};\n mov.b64 c, {%6, %6};\n mov.b64 x, {%4, %5};\n"
        " mul.rn.f32x2 al, al, c;\n fma.rn.f32x2 e, al, x, x;\n mov.b64 {%0, %1}, e;\n}\n"
        : "=f"(e0), "=f"(e1)
        : "f"(al0), "f"(al1), "f"(x0), "f"(x1), "f"(-MGK_LN2F));
}

__device__ __forceinline__ float exp2_pair(float ah, float al) {
    const float e = mgk_ex2(-ah);
    return __fmaf_rn(__fmul_rn(-al, MGK_LN2F), e, e);
}

__device__ __forceinline__ float rcp_approx(float x) {
    float y;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

__device__ __forceinline__ float rsqrt_approx(float x) {
    float y;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// (a0, a1) += (e0, e1) * f as one packed FP32 FMA (fma.rn.f32x2): each half
// is the correctly rounded a + e * f, bitwise the scalar __fmaf_rn.
__device__ __forceinline__ void fma2_bcast(float& a0, float& a1, float e0, float e1, float f) {
    asm("{\n .reg .b64 a, e, f;\n mov.b64 a, {%0, %1};\n mov.b64 e, {%2, %3};\n mov.b64 f, {%4, %4};\n"
        " fma.rn.f32x2 a, e, f, a;\n mov.b64 {%0, %1}, a;\n}\n"
        : "+f"(a0), "+f"(a1)
        : "f"(e0), "f"(e1), "f"(f));
}

// acc += e * f when a < t: one compare and one predicated FFMA.
__device__ __forceinline__ void fma_if_less(float& acc, float a, float t, float e, float f) {
    asm("{\n .reg .pred p;\n setp.lt.f32 p, %1, %2;\n @p fma.rn.f32 %0, %3, %4, %0;\n}\n"
        : "+f"(acc)
        : "f"(a), "f"(t), "f"(e), "f"(f));
}

// Does some column of a regular 128-column block lie within the ambiguity
// band of a row?  For the row, in-disc columns satisfy dx^2 < s2 with
// s2 = 9h^2 - dy^2 (squared half-chord); the FP32 decision a_j < T_i can
// differ from the exact one only for columns with |dx^2 - s2| < eps_d2, i.e.
// within eps_d2 / (2 s) of a crossing x = px +- s.  pc0 = (px - cx_0) / cs in
// columns; margins cover the float error of the crossing positions.  Returns
// two bits: bit 0 for columns 0-63 (warp column half 0), bit 1 for 64-127.
__device__ __forceinline__ unsigned amb_row(float s2, float eps_d2, float pc0, float inv_cs) {
    const float r = rsqrt_approx(fmaxf(s2, 1e-30f));
    const float sc = s2 * r * inv_cs;  // half-chord in columns (0 when s2 <= 0)
    const float wc = __fmaf_rn(eps_d2 * 0.5f * inv_cs, r, __fmaf_rn(4e-7f, sc + fabsf(pc0), 1e-6f));
    if (s2 < -eps_d2) return 0u;
    if (wc > 0.25f) return 3u;
    const float fp = pc0 + sc, fm = pc0 - sc;
    const bool np = fabsf(fp - rintf(fp)) < wc, nm = fabsf(fm - rintf(fm)) < wc;
    // a crossing near column position f concerns half 0 if f <= 64, half 1 if f >= 63
    const unsigned b0 = (np && fp >= -1.0f && fp <= 64.0f) || (nm && fm >= -1.0f && fm <= 64.0f);
    const unsigned b1 = (np && fp >= 63.0f && fp <= 128.0f) || (nm && fm >= 63.0f && fm <= 128.0f);
    return b0 | (b1 << 1);
}

// A mini-batch takes its points from kNCur cursors over equal consecutive
// parts of the item's candidate range (round robin, up to kMB / kNCur from
// each, then whatever is left).  With several cursors the points of one batch
// come from bin rows spread over the candidate window, which evens the eight
// warps' phase-B work per batch; with one, neighbouring points share their
// branches in phase A.  Since three CTAs share an SM (the others issue while
// one waits at a batch barrier) one cursor is the faster: 8.01 ms on the C1
// raster against 8.34 ms with two and 8.42 ms with eight.
#ifndef MGK_DENSITY_NCUR
#define MGK_DENSITY_NCUR 1
#endif
constexpr int kNCur = MGK_DENSITY_NCUR;
struct BatchCur {
    long long by, seq, pos, end;  // bin row, its offset in the block's sequence, next and end candidate
    long long sb, len;            // the current row's range of the index
};

// Cursor c of an item: candidates [k0 + (k1 - k0) c / kNCur, ...) of the block's sequence.
__device__ __forceinline__ void cur_init(const DParams& P, const BlockGeom& G, const Item& it, int c, BatchCur& s) {
    const long long k0 = it.k0, k1 = it.k1;
    s.by = G.by0;
    s.seq = 0;
    s.pos = k0 + (k1 - k0) * c / kNCur;
    s.end = k0 + (k1 - k0) * (c + 1) / kNCur;
    s.sb = s.len = 0;
    if (G.any) {
        int64_t sb, len;
        row_span(P, G, G.by0, sb, len);
        s.sb = sb;
        s.len = len;
    }
}

// Up to `limit` more candidates from cursor s into dst[m..] (one bulk copy per
// row segment, completing on bar); returns the new m.
__device__ __forceinline__ int cur_take(const DParams& P, const BlockGeom& G, BatchCur& s, int m, int limit,
                                        MgkPt* dst, uint64_t* bar) {
    while (m < limit && s.by <= G.by1 && s.pos < s.end) {
        const long long lo = s.pos > s.seq ? s.pos : s.seq;
        const long long hi = (s.seq + s.len) < s.end ? (s.seq + s.len) : s.end;
        if (lo < hi) {
            const int n = (int)((limit - m) < (hi - lo) ? (limit - m) : (hi - lo));
            bulk_g2s(dst + m, P.pts + s.sb + (lo - s.seq), (unsigned)(n * sizeof(MgkPt)), bar);
            s.pos = lo + n;
            m += n;
        } else {
            s.seq += s.len;
            if (++s.by <= G.by1) {
                int64_t sb, len;
                row_span(P, G, s.by, sb, len);
                s.sb = sb;
                s.len = len;
            }
        }
    }
    return m;
}

// Stages the next mini-batch of the item into dst (called by one thread; the
// cursors live in shared memory).  Returns the batch size (0 at the end).
__device__ __forceinline__ int fill_batch(const DParams& P, const BlockGeom& G, BatchCur* cur, MgkPt* dst,
                                          uint64_t* bar) {
    if (!G.any) return 0;
    int m = 0;
    for (int c = 0; c < kNCur; c++) m = cur_take(P, G, cur[c], m, m + kMB / kNCur, dst, bar);
    for (int c = 0; c < kNCur && m < kMB; c++) m = cur_take(P, G, cur[c], m, kMB, dst, bar);
    if (m > 0) mbar_arrive_tx(bar, (unsigned)(m * sizeof(MgkPt)));
    return m;
}

// Dynamic shared memory of k_density (bytes): the staged points and the
// factor tables, 128 column and 64 row entries per point.  A warp stores 32
// consecutive entries of one point at a time, so the tables need no padding
// against bank conflicts, and three CTAs fit on an SM.  The per-cell Kahan
// accumulators are in tensor memory.
constexpr int kFStrideC = 128;  // column table, floats per point
constexpr int kFStride = 64;    // row tables, floats per point
constexpr size_t kSmemStage = 2 * kMB * sizeof(MgkPt);
constexpr size_t kSmemColTab = (size_t)kMB * kFStrideC * sizeof(float);
constexpr size_t kSmemRowTab = (size_t)kMB * kFStride * sizeof(float);
constexpr size_t kDensitySmem = kSmemStage + kSmemColTab + 2 * kSmemRowTab;

// Resident CTAs per SM: three (24 warps) need at most 80 registers per
// thread and about 72 KB of shared memory per CTA; with two (128 registers)
// the C1 kernel took 9.58 ms against 8.72 ms.
#ifndef MGK_DENSITY_MIN_CTAS
#define MGK_DENSITY_MIN_CTAS 3
#endif

// Table entry of column j (row i) of batch point q.
__device__ __forceinline__ int col_slot(int q, int j) { return q * kFStrideC + j; }
__device__ __forceinline__ int row_slot(int q, int i) { return q * kFStride + i; }
// Phase A builds the cutoff thresholds and ambiguity flags of a row only when
// a sub-block that sums the point is partial in that row's warp row (fully
// inside sub-blocks read neither).
#ifndef MGK_DENSITY_ROWSKIP
#define MGK_DENSITY_ROWSKIP 1
#endif
// Phase B takes a half-batch's fully-inside points in one loop and its
// partial ones in another, and decides the Kahan flush once per half-batch.
#ifndef MGK_DENSITY_SPLITLOOP
#define MGK_DENSITY_SPLITLOOP 1
#endif

// Warp sub-blocks: 32 x 32 cells, 2 warp rows x 4 warp columns; lanes own
// 4 rows and 8 contiguous columns (the 4 lanes of a row read 128 contiguous
// bytes of a column table).  A disc's edge crosses fewer square sub-blocks
// than 16 x 64 ones (9.57 against 9.71 ms on the C1 raster).
constexpr int kWR = 32;           // rows of a warp's sub-block
constexpr int kWC = 32;           // columns of a warp's sub-block
constexpr int kNWC = kBC / kWC;   // warps across the block (4)
constexpr int kLC = 4;            // lanes across a sub-block
constexpr int kE2 = 4;            // offset of a lane's second group of 4 columns
static_assert(kBR == 2 * kWR && kNWC == 4 && kThreads == 256, "phase A assumes 2 x 4 warps of 32 x 32 cells");

// Block column of cell j (0..7) of lane column tc in warp column wc.
__device__ __forceinline__ int lane_col(int wc, int tc, int j) { return wc * 32 + tc * 8 + j; }

// The thread's FP32 partial sums into its Kahan-compensated accumulators in
// tensor memory (sum at tS, compensation at tC), then zeroed.
__device__ __forceinline__ void flush_partials(unsigned tS, unsigned tC, float (&part)[32]) {
    __syncwarp();
    tmem_wait_st();  // the previous flush's stores have landed
#pragma unroll
    for (int c = 0; c < 4; c++) {
        float sv[8], cv[8];
        tmem_ld8(tS + 8u * c, sv);
        tmem_ld8(tC + 8u * c, cv);
        tmem_wait_ld(sv, cv);
#pragma unroll
        for (int u = 0; u < 8; u += 2) {
            kahan_add2(sv[u], sv[u + 1], cv[u], cv[u + 1], part[c * 8 + u], part[c * 8 + u + 1]);
            part[c * 8 + u] = 0.0f;
            part[c * 8 + u + 1] = 0.0f;
        }
        tmem_st8(tS + 8u * c, sv);
        tmem_st8(tC + 8u * c, cv);
    }
}

// One work item: the gather of the candidate range [it.k0, it.k1) of one
// 64 x 128 block (the body of k_density and of the multi-job k_density_jobs).
template <bool VARH, bool COUNT>
__device__ __forceinline__ void density_item(const DParams& P, const Item it) {
    extern __shared__ __align__(128) unsigned char dsm[];
    MgkPt* stage = reinterpret_cast<MgkPt*>(dsm);                                    // [2][kMB]
    float* colE = reinterpret_cast<float*>(dsm + kSmemStage);                   // [kMB][kFStrideC] E_j
    float* rowF = reinterpret_cast<float*>(dsm + kSmemStage + kSmemColTab);     // [kMB][kFStride] F_i
    float* rowG = reinterpret_cast<float*>(dsm + kSmemStage + kSmemColTab + kSmemRowTab);  // [kMB][kFStride] G_i
    __shared__ __align__(8) uint64_t mbar[2];
    __shared__ unsigned s_tmem;  // TMEM base of the block's Kahan accumulators
    __shared__ __align__(16) unsigned long long rowflag[kMB][2];  // per column half: 64 row bits
    __shared__ unsigned char procmask[kMB];  // warp w processes the point
    __shared__ unsigned char fullmask[kMB];  // every cell of warp w's sub-block is inside the cutoff
    __shared__ float s_cxh[kBC], s_cxl[kBC], s_cxg[kBC], s_cyh[kBR], s_cyl[kBR], s_cyg[kBR];
    __shared__ BatchCur s_cur[kNCur];  // the item's candidate cursors
    __shared__ int s_nm;               // size of the batch being staged
    __shared__ int s_load[2][8];       // per batch buffer: points warp w sums (phase B)

    const BlockGeom G = block_geom(P, it.bx, it.by);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int wr = warp / kNWC, wc = warp % kNWC;  // warp sub-block: rows wr*kWR.., cols wc*kWC..
    // lane micro-tile: rows tr*4.. (4) and the 8 columns lane_col(wc, tc, 0..7)
    // (contiguous in 32 x 32 sub-blocks: the 4 lanes of a row read 128
    // contiguous bytes of E; in 16 x 64 ones two groups of 4, 32 apart)
    const int tr = lane / kLC, tc = lane % kLC;

    // cell centres of the block: global floats and their quantum split
    bool regular = true;
    if (tid < kBC) {
        const float cx = mgk_cell_x(P.xll, P.cs, G.c0 + tid);
        s_cxg[tid] = cx;
        mgk_qsplit(cx, P.qexp, s_cxh[tid], s_cxl[tid]);
        const float cx0 = mgk_cell_x(P.xll, P.cs, G.c0);
        regular = ((double)cx - (double)cx0) == (double)tid * P.cs;
    } else if (tid < kBC + kBR) {
        const float cy = mgk_cell_y(P.yll, P.cs, P.g_nrows, G.r0 + tid - kBC);
        s_cyg[tid - kBC] = cy;
        mgk_qsplit(cy, P.qexp, s_cyh[tid - kBC], s_cyl[tid - kBC]);
    }
    if (tid == 0) {
        mbar_init(&mbar[0], 1);
        mbar_init(&mbar[1], 1);
        fence_mbar_init();
    }
    if (tid < 16) s_load[tid >> 3][tid & 7] = 0;
    __syncwarp();
    if (warp == 0) tmem_alloc(&s_tmem);
    tmem_fence_before();
    regular = __syncthreads_and(regular);
    tmem_fence_after();
    // Kahan sum and compensation of the thread's 32 cells (cell k = i * 8 + j
    // at column k of tS and of tC)
    const unsigned tS = s_tmem + ((32u * (unsigned)(warp & 3)) << 16) + 64u * (unsigned)(warp >> 2);
    const unsigned tC = tS + 32u;
    {
        const float z[8] = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
#pragma unroll
        for (int c = 0; c < 4; c++) {
            tmem_st8(tS + 8u * c, z);
            tmem_st8(tC + 8u * c, z);
        }
    }
    const float inv_cs = 1.0f / (float)P.cs;

    // validity of the lane's 32 cells (inside the tile and not NoData); bit
    // i*8+j.  Mask rows (and output rows, in the epilogue) go 8 cells, two
    // 16-byte vectors, at a time where the raster rows keep 16-byte alignment.
    unsigned valid = 0;
    {
    const bool vec = (P.nc & 3) == 0 && (reinterpret_cast<uintptr_t>(P.mask) & 15u) == 0;
    const int lc0 = lane_col(wc, tc, 0);
#pragma unroll
    for (int i = 0; i < 4; i++) {
        const int r = wr * kWR + tr * 4 + i;
        if (r >= G.nrow) continue;
        const int64_t o = (G.r0 + r - P.row0) * P.nc + (G.c0 + lc0 - P.col0);
        if (P.mbits) {
            // one byte holds the lane's 8 columns (lc0 and the tile's block
            // origins are multiples of 8); bits past the tile's edge are dropped
            const unsigned b = P.mbits[(G.r0 + r - P.row0) * P.mbstride + ((G.c0 - P.col0 + lc0) >> 3)];
            const int nv = min(8, max(0, G.ncol - lc0));
            valid |= (b & ((1u << nv) - 1u)) << (i * 8);
        } else if (P.mask && vec && lc0 + 8 <= G.ncol) {
            const float4 a = __ldg(reinterpret_cast<const float4*>(P.mask + o));
            const float4 b = __ldg(reinterpret_cast<const float4*>(P.mask + o + 4));
            const float m8[8] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
#pragma unroll
            for (int j = 0; j < 8; j++) valid |= (unsigned)(m8[j] != P.nodata) << (i * 8 + j);
        } else {
#pragma unroll
            for (int j = 0; j < 8; j++) {
                bool v = lc0 + j < G.ncol;
                if (v && P.mask) v = P.mask[o + j] != P.nodata;
                valid |= (unsigned)v << (i * 8 + j);
            }
        }
    }
    }
    // A block whose cells are all NoData gathers no candidates: its output
    // is NoData throughout (the reference skips NoData cells before any sum,
    // kde_kernel_kdtr.cu:426-428).
    const bool any_valid = __syncthreads_or(valid != 0u);

    float part[32];
#pragma unroll
    for (int k = 0; k < 32; k++) part[k] = 0.0f;
    unsigned long long cnt = 0;
    unsigned pc = 0;  // points processed by this warp (warp-uniform)

    // phase-A skip tests: thread tid tests point qa = tid / 8 (and qa + 32)
    // against sub-block ka = tid % 8
    const int qa = tid >> 3, ka = tid & 7;
    const int sk_wr = ka / kNWC, sk_wc = ka % kNWC;
    const bool sk_on = (sk_wr * kWR < G.nrow) && (sk_wc * kWC < G.ncol);
    const int sk_c0 = sk_wc * kWC, sk_c1 = min(sk_wc * kWC + kWC - 1, G.ncol - 1);
    const int sk_r0 = sk_wr * kWR, sk_r1 = min(sk_wr * kWR + kWR - 1, G.nrow - 1);

    if (tid == 0) {
        for (int c = 0; c < kNCur; c++) cur_init(P, G, it, c, s_cur[c]);
        s_nm = any_valid ? fill_batch(P, G, s_cur, &stage[0], &mbar[0]) : 0;
    }
    __syncthreads();
    int m = s_nm;
    unsigned phase0 = 0, phase1 = 0;
    int buf = 0;
    // Two block barriers per batch: after the factor tables (which also
    // shares a staging wait that ran out) and after the sums.  The next
    // batch is staged during the sums, by the warp with the fewest points to
    // sum, so the serial fill is off the critical path.
    bool aborted = false;
    unsigned abort_par = 0;
    while (m > 0) {
        const unsigned par = buf ? phase1 : phase0;
        const bool ok = mbar_wait(&mbar[buf], par);  // every thread; bounded
        if (!ok) atomicExch(P.err, 1ull);
        if (buf) phase1 ^= 1u;
        else phase0 ^= 1u;
        const MgkPt* st = stage + buf * kMB;

        // ---------------- phase A ----------------
        // Warp w takes points 4w..4w+3 and 32+4w..32+4w+3.  For each group of
        // four, lane (k, ka) = (lane / 8, lane % 8) tests point k against
        // sub-block ka; then the warp builds the tables of the four points one
        // at a time, every lane one column of each summed 32-column group and
        // one row of each summed warp row (the warp takes one point's
        // branches, and its stores fill 32 consecutive entries).
#pragma unroll 1
        for (int hq = 0; hq < kMB / 32; hq++) {
            const int pq = qa + 32 * hq;
            const bool act = ok && pq < m;
            bool proc = false, full = false;
            if (act && sk_on) {
                const MgkPt r = st[pq];
                const float cutf = VARH ? 9.0f * r.hh : P.cutf;
                // distance from the point to the sub-block rectangle of cell centres
                const float dxl = __fadd_rn(__fsub_rn(s_cxh[sk_c0], r.xh), __fsub_rn(s_cxl[sk_c0], r.xl));
                const float dxr = __fadd_rn(__fsub_rn(r.xh, s_cxh[sk_c1]), __fsub_rn(r.xl, s_cxl[sk_c1]));
                const float dyt = __fadd_rn(__fsub_rn(r.yh, s_cyh[sk_r0]), __fsub_rn(r.yl, s_cyl[sk_r0]));
                const float dyb = __fadd_rn(__fsub_rn(s_cyh[sk_r1], r.yh), __fsub_rn(s_cyl[sk_r1], r.yl));
                const float ddx = fmaxf(0.0f, fmaxf(dxl, dxr));
                const float ddy = fmaxf(0.0f, fmaxf(dyt, dyb));
                proc = ddx * ddx + ddy * ddy < cutf * 1.0001f;
                // farthest corner well inside the cutoff: no cell of the sub-block needs the test
                const float fx = fmaxf(fabsf(dxl), fabsf(dxr)), fy = fmaxf(fabsf(dyt), fabsf(dyb));
                full = fx * fx + fy * fy < cutf * 0.9999f;
            }
            const unsigned bal = __ballot_sync(0xffffffffu, proc);
            const unsigned balf = __ballot_sync(0xffffffffu, full);
            if (lane < 8) {
                // this warp's points (4) that sub-block warp `lane` sums
                const int nl = __popc(bal & (0x01010101u << lane));
                if (nl) atomicAdd(&s_load[buf][lane], nl);
            }
            if (ka == 0) {
                procmask[pq] = (unsigned char)((bal >> (8 * (qa & 3))) & 0xffu);
                fullmask[pq] = (unsigned char)((balf >> (8 * (qa & 3))) & 0xffu);
            }
#pragma unroll 1
            for (int k = 0; k < 4; k++) {
                // the sub-blocks that sum point pk: bit b is sub-block (b / 4, b % 4).
                // Only their column groups and warp rows of the tables are
                // built; the other entries are never read (the warps that
                // would read them skip the point)
                const unsigned pb = (bal >> (8 * k)) & 0xffu;
                if (!pb) continue;
                // sub-blocks that sum the point with the cutoff test (all of them in the counting variant)
                const unsigned pbp = (MGK_DENSITY_ROWSKIP && !COUNT) ? pb & ~((balf >> (8 * k)) & 0xffu) : pb;
                const int pk = 4 * warp + k + 32 * hq;
                const MgkPt r = st[pk];
                float k2h, k2l, cutf, epsd2;
                if (VARH) {
                    k2h = r.k2h;
                    k2l = r.k2l;
                    cutf = 9.0f * r.hh;
                    epsd2 = r.hh * (4.0f * kAmbEps / (float)MGK_LOG2E);
                } else {
                    k2h = P.k2h;
                    k2l = P.k2l;
                    cutf = P.cutf;
                    epsd2 = P.epsd2;
                }
                // the summed column groups two at a time (the first two left,
                // whichever they are), two entries in packed FP32; a last odd
                // group alone
                unsigned ub = (pb | (pb >> 4)) & 0xfu;
#pragma unroll
                for (int h2 = 0; h2 < 2; h2++) {
                    if (!ub) break;
                    const int u0 = __ffs(ub) - 1;
                    ub &= ub - 1u;
                    const int j0 = lane + 32 * u0;
                    if (ub) {
                        const int u1 = __ffs(ub) - 1;
                        ub &= ub - 1u;
                        const int j1 = lane + 32 * u1;
                        float e0, e1, d20, d21;
                        exp2_pair2(__fsub_rn(r.xh, s_cxh[j0]), __fsub_rn(r.xh, s_cxh[j1]), __fsub_rn(r.xl, s_cxl[j0]),
                                   __fsub_rn(r.xl, s_cxl[j1]), k2h, k2l, e0, e1, d20, d21);
                        colE[col_slot(pk, j0)] = e0;
                        colE[col_slot(pk, j1)] = e1;
                    } else {
                        float ah, al, d2;
                        exponent_pair(__fsub_rn(r.xh, s_cxh[j0]), __fsub_rn(r.xl, s_cxl[j0]), k2h, k2l, ah, al, d2);
                        colE[col_slot(pk, j0)] = exp2_pair(ah, al);
                    }
                }
                const float pc0 = __fadd_rn(__fsub_rn(r.xh, s_cxh[0]), __fsub_rn(r.xl, s_cxl[0])) * inv_cs;
                unsigned flw[2][2] = {{0u, 0u}, {0u, 0u}};  // [column half][warp row]: row bits
                // row factors of both warp rows (packed when both are summed)
                float fbv[2], d2v[2];
                if ((pb & 0xfu) && (pb >> 4)) {
                    exp2_pair2(__fsub_rn(r.yh, s_cyh[lane]), __fsub_rn(r.yh, s_cyh[lane + 32]),
                               __fsub_rn(r.yl, s_cyl[lane]), __fsub_rn(r.yl, s_cyl[lane + 32]), k2h, k2l, fbv[0],
                               fbv[1], d2v[0], d2v[1]);
                } else {
                    const int i = (pb & 0xfu) ? lane : lane + 32;
                    float bh, bl, d2;
                    exponent_pair(__fsub_rn(r.yh, s_cyh[i]), __fsub_rn(r.yl, s_cyl[i]), k2h, k2l, bh, bl, d2);
                    fbv[0] = fbv[1] = exp2_pair(bh, bl);
                    d2v[0] = d2v[1] = d2;
                }
#pragma unroll
                for (int v = 0; v < 2; v++) {
                    const bool row_on = (pb >> (4 * v)) & 0xfu;  // warp-uniform
                    if (!row_on) continue;
                    const int i = lane + 32 * v;
                    const float fb = fbv[v], d2 = d2v[v];
                    rowF[row_slot(pk, i)] = __fmul_rn(r.wk, fb);
                    // no partial sub-block reads the row's G
                    if (!((pbp >> (4 * v)) & 0xfu)) continue;
                    // a_j < cutl - b_i  <=>  E_j > G_i = 2^-cutl / 2^-b_i (2^-x is decreasing);
                    // G = inf for rows off the disc (2^-b_i flushed to zero)
                    rowG[row_slot(pk, i)] = __fmul_rn(P.gcut, rcp_approx(fb));
                    const float s2 = cutf - d2;
                    const unsigned a = regular ? amb_row(s2, epsd2, pc0, inv_cs) : (s2 >= -epsd2 ? 3u : 0u);
                    flw[0][v] = __ballot_sync(0xffffffffu, a & 1u);
                    flw[1][v] = __ballot_sync(0xffffffffu, a >> 1);
                }
                if (lane == 0) {
                    rowflag[pk][0] = ((unsigned long long)flw[0][1] << 32) | flw[0][0];
                    rowflag[pk][1] = ((unsigned long long)flw[1][1] << 32) | flw[1][0];
                }
            }
        }
        if (__syncthreads_or(!ok)) {
            // a staging wait ran out: the batch's copy is the only one in flight
            aborted = true;
            abort_par = par;
            break;
        }

        // ---------------- phase B ----------------
        {
            // stage the next batch: the warp with the fewest points to sum
            // (lowest index on ties) fills; the buffer's last readers were
            // the previous batch's sums, before that batch's end barrier
            int filler = 0, least = s_load[buf][0];
#pragma unroll
            for (int w = 1; w < 8; w++)
                if (s_load[buf][w] < least) {
                    least = s_load[buf][w];
                    filler = w;
                }
            if (warp == filler && lane == 0) s_nm = fill_batch(P, G, s_cur, &stage[(buf ^ 1) * kMB], &mbar[buf ^ 1]);
            if (tid == 32 * ((filler + 1) & 7)) {
                // the other buffer's counts were last read before the previous end barrier
#pragma unroll
                for (int w = 0; w < 8; w++) s_load[buf ^ 1][w] = 0;
            }
            // the batch in halves of 32 points, one lane per point
#pragma unroll 1
            for (int hq = 0; hq < kMB / 32; hq++) {
                // this warp's processed, fully-inside and flagged points of the batch as bit masks
                const int pl = lane + 32 * hq;  // this lane's point of the half
                const bool lv = pl < m;
                const bool pm = lv && ((procmask[pl] >> warp) & 1u);
                const bool fm = lv && ((fullmask[pl] >> warp) & 1u);
                // the 32 rows of the warp in its column half (wc / 2), point pl
                const unsigned myflag =
                    lv ? reinterpret_cast<const unsigned*>(&rowflag[0][0])[pl * 4 + (wc >> 1) * 2 + wr] : 0u;
                unsigned todo = __ballot_sync(0xffffffffu, pm);
                const unsigned fullb = __ballot_sync(0xffffffffu, pm && fm);
                const unsigned ambb = __ballot_sync(0xffffffffu, pm && myflag != 0u);
#if MGK_DENSITY_SPLITLOOP
                // the partials hold at most 32 points: flush before a half that would exceed that
                const unsigned nh = (unsigned)__popc(todo);
                if (pc + nh > 32u) {
                    flush_partials(tS, tC, part);
                    pc = 0;
                }
                pc += nh;
                // fully-inside points first, then the partial ones; the counting
                // variant takes the same order (through the compare path), so
                // its raster is bitwise the plain variant's
                unsigned rest = todo & ~fullb;
                todo &= fullb;
                if (!COUNT) {
                    while (todo) {
                        const int q = __ffs(todo) - 1, qq = q + 32 * hq;
                        todo &= todo - 1u;
                        const float* pE = colE + col_slot(qq, lane_col(wc, tc, 0));
                        const float* pE2 = pE + kE2;
                        const float* pF = rowF + row_slot(qq, wr * kWR + tr * 4);
                        const float4 e4a = *reinterpret_cast<const float4*>(pE);
                        const float4 e4b = *reinterpret_cast<const float4*>(pE2);
                        const float4 f4 = *reinterpret_cast<const float4*>(pF);
                        const float ce[8] = {e4a.x, e4a.y, e4a.z, e4a.w, e4b.x, e4b.y, e4b.z, e4b.w};
                        const float rv[4] = {f4.x, f4.y, f4.z, f4.w};
#pragma unroll
                        for (int i = 0; i < 4; i++)
#pragma unroll
                            for (int j = 0; j < 8; j += 2)
                                fma2_bcast(part[i * 8 + j], part[i * 8 + j + 1], ce[j], ce[j + 1], rv[i]);
                    }
                    todo = rest;
                    rest = 0u;
                }
#endif
                for (;;) {  // one pass; with the split loops, a second over `rest`
                    while (todo) {
                        const int q = __ffs(todo) - 1, qq = q + 32 * hq;
                        todo &= todo - 1u;
                        const float* pE = colE + col_slot(qq, lane_col(wc, tc, 0));
                        const float* pE2 = pE + kE2;
                        const float* pF = rowF + row_slot(qq, wr * kWR + tr * 4);
                        const float4 e4a = *reinterpret_cast<const float4*>(pE);
                        const float4 e4b = *reinterpret_cast<const float4*>(pE2);
                        const float4 f4 = *reinterpret_cast<const float4*>(pF);
                        const float ce[8] = {e4a.x, e4a.y, e4a.z, e4a.w, e4b.x, e4b.y, e4b.z, e4b.w};
                        const float rv[4] = {f4.x, f4.y, f4.z, f4.w};
                        // (with the split loops no fully-inside point is left here)
                        if (!COUNT && !MGK_DENSITY_SPLITLOOP && ((fullb >> q) & 1u)) {
                            // the whole sub-block is inside the cutoff: one FFMA per cell
#pragma unroll
                            for (int i = 0; i < 4; i++)
#pragma unroll
                                for (int j = 0; j < 8; j++) part[i * 8 + j] = __fmaf_rn(ce[j], rv[i], part[i * 8 + j]);
                        } else {
                            const float4 g4 = *reinterpret_cast<const float4*>(rowG + row_slot(qq, wr * kWR + tr * 4));
                            const float rg[4] = {g4.x, g4.y, g4.z, g4.w};
                            unsigned inm = 0;
                            if (COUNT) {
#pragma unroll
                                for (int i = 0; i < 4; i++)
#pragma unroll
                                    for (int j = 0; j < 8; j++) {
                                        const bool in = rg[i] < ce[j];
                                        if (in) part[i * 8 + j] = __fmaf_rn(ce[j], rv[i], part[i * 8 + j]);
                                        inm |= (unsigned)in << (i * 8 + j);
                                    }
                            } else {
#pragma unroll
                                for (int i = 0; i < 4; i++)
#pragma unroll
                                    for (int j = 0; j < 8; j++) fma_if_less(part[i * 8 + j], rg[i], ce[j], ce[j], rv[i]);
                            }
                            if ((ambb >> q) & 1u) {
                                // some row of this sub-block has a column in the cutoff band: exact FP64 re-decision
                                const unsigned fl = (__shfl_sync(0xffffffffu, myflag, q) >> (tr * 4)) & 0xfu;
                                if (fl) {
                                    const MgkPt r = st[qq];
                                    const float px = r.xh + r.xl, py = r.yh + r.yl;
                                    const double cut = VARH ? MGK_CUT * (double)r.hh : P.cut_d2;
#pragma unroll
                                    for (int i = 0; i < 4; i++) {
                                        if (!((fl >> i) & 1u)) continue;
#pragma unroll
                                        for (int j = 0; j < 8; j++) {
                                            const bool ex = mgk_d2_exact(px, py, s_cxg[lane_col(wc, tc, j)],
                                                                         s_cyg[wr * kWR + tr * 4 + i]) < cut;
                                            const bool fi = rg[i] < ce[j];
                                            if (ex != fi) {
                                                const float t = __fmul_rn(ce[j], rv[i]);
                                                part[i * 8 + j] = __fadd_rn(part[i * 8 + j], ex ? t : -t);
                                                if (COUNT) inm ^= 1u << (i * 8 + j);
                                            }
                                        }
                                    }
                                }
                            }
                            if (COUNT) cnt += __popc(inm & valid);
                        }
#if !MGK_DENSITY_SPLITLOOP
                        pc++;
                        if ((pc & 31u) == 0) flush_partials(tS, tC, part);  // 32-point partials
#endif
                    }
#if MGK_DENSITY_SPLITLOOP
                    if (!rest) break;
                    todo = rest;
                    rest = 0u;
#else
                    break;
#endif
                }
            }
        }
        __syncthreads();  // factor tables, s_nm and stage[buf] are reused next
        m = s_nm;
        buf ^= 1;
    }
    __syncwarp();
    tmem_wait_st();
    if (aborted) {
        // give the outstanding copy a second bounded wait before the CTA (and
        // its shared memory) goes away; release the tensor memory
        if (tid == 0) mbar_wait(&mbar[buf], abort_par);
        tmem_fence_before();
        __syncthreads();
        if (warp == 0) {
            tmem_fence_after();
            tmem_dealloc(s_tmem);
        }
        return;
    }

    // epilogue: FP64 result = (s - c) * normalisation
    const double norm = VARH ? 1.0 : P.k0;
#pragma unroll
    for (int q8 = 0; q8 < 4; q8++) {
        float ss[8], cc[8];
        __syncwarp();
        tmem_ld8(tS + 8u * q8, ss);
        tmem_ld8(tC + 8u * q8, cc);
        tmem_wait_ld(ss, cc);
#pragma unroll
        for (int u = 0; u < 8; u++) kahan_add(ss[u], cc[u], part[q8 * 8 + u]);
        // row q8 of the lane's micro-tile: cells k = q8 * 8 + u, columns ec0 + u
        const int r = wr * kWR + tr * 4 + q8, ec0 = lane_col(wc, tc, 0);
        if (r >= G.nrow) continue;
        if (it.slot >= 0) {
            double* d = P.scratch + (size_t)it.slot * kCells + r * kBC + ec0;
#pragma unroll
            for (int u = 0; u < 8; u++)
                if (ec0 + u < G.ncol) d[u] = ((double)ss[u] - (double)cc[u]) * norm;
        } else {
            float* d = P.out + (G.r0 + r - P.row0) * P.nc + (G.c0 + ec0 - P.col0);
            float f[8];
#pragma unroll
            for (int u = 0; u < 8; u++)
                f[u] = ((valid >> (q8 * 8 + u)) & 1u) ? (float)(((double)ss[u] - (double)cc[u]) * norm) : P.nodata;
            const bool vec = (P.nc & 3) == 0 && (reinterpret_cast<uintptr_t>(P.out) & 15u) == 0;
            if (vec && ec0 + 8 <= G.ncol) {
                *reinterpret_cast<float4*>(d) = make_float4(f[0], f[1], f[2], f[3]);
                *reinterpret_cast<float4*>(d + 4) = make_float4(f[4], f[5], f[6], f[7]);
            } else {
#pragma unroll
                for (int u = 0; u < 8; u++)
                    if (ec0 + u < G.ncol) d[u] = f[u];
            }
        }
    }
    tmem_fence_before();
    __syncthreads();
    if (warp == 0) {
        tmem_fence_after();
        tmem_dealloc(s_tmem);
    }
    if (COUNT) {
        for (int o = 16; o; o >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
        if (lane == 0 && cnt) atomicAdd(P.evals, cnt);
    }
}

template <bool VARH, bool COUNT>
__global__ void __launch_bounds__(kThreads, MGK_DENSITY_MIN_CTAS) k_density(DParams P) {
    // the last CTA to start tells a stream waiting on the flag (the next
    // band's launch) that this launch's tail has begun
    if (P.tail_flag && blockIdx.x == gridDim.x - 1 && threadIdx.x == 0) atomicExch(P.tail_flag, 1u);
    density_item<VARH, COUNT>(P, P.items[blockIdx.x]);
}

// Each CTA copies its job's parameters (device memory) into shared memory
// once; the item loop then reads them from there.
__device__ __forceinline__ void load_job(const DParams* jobs, int j, DParams& dst) {
    static_assert(sizeof(DParams) % 8 == 0, "DParams is copied in 8-byte words");
    const unsigned long long* src = reinterpret_cast<const unsigned long long*>(jobs + j);
    unsigned long long* d = reinterpret_cast<unsigned long long*>(&dst);
    for (int i = threadIdx.x; i < (int)(sizeof(DParams) / 8); i += blockDim.x) d[i] = src[i];
    __syncthreads();
}

// Several tiles (of one or several indexes and rasters) in one launch: item
// it belongs to job it.pad, whose parameters are jobs[it.pad].
template <bool VARH, bool COUNT>
__global__ void __launch_bounds__(kThreads, MGK_DENSITY_MIN_CTAS) k_density_jobs(const DParams* __restrict__ jobs,
                                                                                 const Item* __restrict__ items) {
    __shared__ __align__(16) DParams sP;
    const Item it = items[blockIdx.x];
    load_job(jobs, it.pad, sP);
    density_item<VARH, COUNT>(sP, it);
}


// Plain FP64 form: same blocks, work items and candidate lists; per pair an
// exact FP64 distance, the cutoff, a double exp and a double accumulate.
template <bool VARH>
__global__ void __launch_bounds__(kThreads, 2) k_density_fp64(DParams P) {
    __shared__ MgkPt sp[kStage64];
    const Item it = P.items[blockIdx.x];
    const BlockGeom G = block_geom(P, it.bx, it.by);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int wr = warp >> 1, wc = warp & 1, tr = lane >> 3, tc = lane & 7;
    float cx[8], cy[4];
#pragma unroll
    for (int j = 0; j < 8; j++) cx[j] = mgk_cell_x(P.xll, P.cs, G.c0 + wc * 64 + tc * 8 + j);
#pragma unroll
    for (int i = 0; i < 4; i++) cy[i] = mgk_cell_y(P.yll, P.cs, P.g_nrows, G.r0 + wr * 16 + tr * 4 + i);
    double acc[32];
#pragma unroll
    for (int k = 0; k < 32; k++) acc[k] = 0.0;
    // all-NoData blocks are skipped, as in the FP32 kernel
    bool mine = false;
    for (int k = 0; k < 32 && !mine; k++) {
        const int r = wr * 16 + tr * 4 + (k >> 3), c = wc * 64 + tc * 8 + (k & 7);
        mine = r < G.nrow && c < G.ncol && cell_valid(P, G.r0 + r - P.row0, G.c0 + c - P.col0);
    }
    if (__syncthreads_or(mine) && G.any) {
        int64_t seq = 0;
        for (int64_t by = G.by0; by <= G.by1 && seq < it.k1; by++) {
            int64_t sb, len;
            row_span(P, G, by, sb, len);
            const int64_t lo = mgk_max64(seq, it.k0), hi = mgk_min64(seq + len, it.k1);
            for (int64_t base = lo; base < hi; base += kStage64) {
                const int m = (int)mgk_min64(kStage64, hi - base);
                const int64_t src = sb + (base - seq);
                __syncthreads();
                for (int k = tid; k < m; k += kThreads) sp[k] = P.pts[src + k];
                __syncthreads();
                for (int q = 0; q < m; q++) {
                    const MgkPt p = sp[q];
                    const float px = p.xh + p.xl, py = p.yh + p.yl;
                    const double h2 = VARH ? (double)p.hh : P.h2;
                    const double cut = MGK_CUT * h2;
                    const double m2h = -1.0 / (2.0 * h2);
#pragma unroll
                    for (int i = 0; i < 4; i++)
#pragma unroll
                        for (int j = 0; j < 8; j++) {
                            const double d2 = mgk_d2_exact(px, py, cx[j], cy[i]);
                            if (d2 < cut) acc[i * 8 + j] += exp(d2 * m2h) * (double)p.wk;
                        }
                }
            }
            seq += len;
        }
    }
    const double norm = VARH ? 1.0 : P.k0;
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 8; j++) {
            const int r = wr * 16 + tr * 4 + i, c = wc * 64 + tc * 8 + j;
            if (r >= G.nrow || c >= G.ncol) continue;
            const double v = acc[i * 8 + j] * norm;
            if (it.slot >= 0) {
                P.scratch[(size_t)it.slot * kCells + r * kBC + c] = v;
            } else {
                const int64_t o = (G.r0 + r - P.row0) * P.nc + (G.c0 + c - P.col0);
                P.out[o] = cell_valid(P, G.r0 + r - P.row0, G.c0 + c - P.col0) ? (float)v : P.nodata;
            }
        }
}

// Merge of split blocks: cell value = sum over the block's slots in order.
// Cells [part * kCells / gridDim.y, ...) of the block: a block's cells are
// spread over gridDim.y CTAs, so each thread sums a few cells and the
// launch is not bound by one CTA's sequential loads.
__device__ __forceinline__ void merge_block(const DParams& P, int32_t blk, int s0, int s1) {
    const int per = kCells / (int)gridDim.y, e0 = (int)blockIdx.y * per;
    const int nbx_t = (int)((P.nc + kBC - 1) / kBC);
    const int bxi = blk % nbx_t, byi = blk / nbx_t;
    const int64_t r0 = P.row0 + (int64_t)byi * kBR, c0 = P.col0 + (int64_t)bxi * kBC;
    const int nrow = (int)mgk_min64(kBR, P.row0 + P.nr - r0);
    const int ncol = (int)mgk_min64(kBC, P.col0 + P.nc - c0);
    for (int e = e0 + (int)threadIdx.x; e < e0 + per; e += blockDim.x) {
        const int r = e / kBC, c = e % kBC;
        if (r >= nrow || c >= ncol) continue;
        double v = 0.0;
        for (int s = s0; s < s1; s++) v += P.scratch[(size_t)s * kCells + e];
        const int64_t o = (r0 + r - P.row0) * P.nc + (c0 + c - P.col0);
        P.out[o] = cell_valid(P, r0 + r - P.row0, c0 + c - P.col0) ? (float)v : P.nodata;
    }
}

__global__ void k_merge(DParams P, const int32_t* __restrict__ blocks, const int32_t* __restrict__ slot_begin) {
    merge_block(P, blocks[blockIdx.x], slot_begin[blockIdx.x], slot_begin[blockIdx.x + 1]);
}

// The launch's staging-wait flag into mapped host memory (no copy engine).
__global__ void k_store_flag(const unsigned long long* __restrict__ src, volatile unsigned long long* dst) {
    *dst = *src;
}

// Merges of several jobs: entry b = {job, block, first slot, end slot}.
__global__ void k_merge_jobs(const DParams* __restrict__ jobs, const int4* __restrict__ list) {
    __shared__ __align__(16) DParams sP;
    const int4 m = list[blockIdx.x];
    load_job(jobs, m.x, sP);
    merge_block(sP, m.y, m.z, m.w);
}

template <bool VARH, bool COUNT>
void launch_density(unsigned grid, cudaStream_t s, const DParams& P) {
    cudaFuncSetAttribute(k_density<VARH, COUNT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kDensitySmem);
    // the largest shared-memory carveout: three CTAs of about 75 KB per SM
    cudaFuncSetAttribute(k_density<VARH, COUNT>, cudaFuncAttributePreferredSharedMemoryCarveout,
                         cudaSharedmemCarveoutMaxShared);
    k_density<VARH, COUNT><<<grid, kThreads, kDensitySmem, s>>>(P);
}

template <bool VARH, bool COUNT>
void launch_density_jobs(unsigned grid, cudaStream_t s, const DParams* jobs, const Item* items) {
    cudaFuncSetAttribute(k_density_jobs<VARH, COUNT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)kDensitySmem);
    cudaFuncSetAttribute(k_density_jobs<VARH, COUNT>, cudaFuncAttributePreferredSharedMemoryCarveout,
                         cudaSharedmemCarveoutMaxShared);
    k_density_jobs<VARH, COUNT><<<grid, kThreads, kDensitySmem, s>>>(jobs, items);
}

// Kernel parameters of one tile over one index.
void fill_params(DParams& P, const mgk_index* idx, const mgk_grid* g, int64_t row0, int64_t col0, int64_t nr,
                 int64_t nc, const float* d_mask, float* d_out) {
    P = DParams{};
    P.xll = g->xll;
    P.yll = g->yll;
    P.cs = g->cs;
    P.g_nrows = g->nrows;
    P.row0 = row0;
    P.col0 = col0;
    P.nr = nr;
    P.nc = nc;
    P.nodata = g->nodata;
    P.mask = d_mask;
    P.out = d_out;
    P.pts = idx->pts;
    P.bin_start = idx->bin_start;
    P.ox = idx->ox;
    P.oy = idx->oy;
    P.side = idx->side;
    P.inv_side = 1.0 / idx->side;
    P.nbx = idx->nbx;
    P.nby = idx->nby;
    P.qexp = idx->qexp;
    P.h2 = idx->h2;
    P.k0 = idx->k0;
    P.cut_d2 = idx->cut_d2;
    P.reach = idx->reach;
    const double k2 = idx->k2;
    P.k2h = (float)k2;
    P.k2l = (float)(k2 - (double)P.k2h);
    // log2-unit cutoff: 9 h^2 k2 for fixed h; 4.5 log2(e) for per-point h
    const double cutl = idx->varh ? MGK_CUT * 0.5 * MGK_LOG2E : idx->cut_d2 * k2;
    P.gcut = (float)std::exp2(-cutl);
    P.cutf = (float)idx->cut_d2;
    // ambiguity band in d^2 units: |a - T| < kAmbEps  <=>  |dx^2 - s^2| < kAmbEps / k2 (x2 margin)
    P.epsd2 = (float)(2.0 * (double)kAmbEps / k2);
}

// Work items of one tile from its per-block candidate counts: blocks above K
// candidates are split into items of at most K (about 8 waves of the
// resident CTAs), each split item writing an FP64 partial into its own
// scratch slot.  K depends on this tile alone, so a tile gets the same items
// (and bitwise the same result) alone or batched with others.
struct TilePlan {
    int nbx_t = 0, nby_t = 0;
    std::vector<Item> items;
    std::vector<int32_t> split_blocks, split_begin;
    int32_t nslots = 0;
};

void plan_tile(const int64_t* counts, int nbx_t, int nby_t, int sm_count, int waves, int job, TilePlan& T) {
    const int nblk = nbx_t * nby_t;
    T.nbx_t = nbx_t;
    T.nby_t = nby_t;
    int64_t total = 0;
    for (int b = 0; b < nblk; b++) total += counts[b];
    const int64_t slots_resident = (int64_t)sm_count * 2;
    int64_t K = std::max<int64_t>(2048, total / std::max<int64_t>(1, slots_resident * waves));
    K = (K + kMB - 1) / kMB * kMB;
    T.items.reserve(nblk + 16);
    for (int b = 0; b < nblk; b++) {
        const int64_t c = counts[b];
        const int bxi = b % nbx_t, byi = b / nbx_t;
        if (c <= K) {
            T.items.push_back({bxi, byi, 0, (int32_t)c, -1, job});
        } else {
            T.split_blocks.push_back(b);
            T.split_begin.push_back(T.nslots);
            for (int64_t k = 0; k < c; k += K) {
                T.items.push_back({bxi, byi, (int32_t)k, (int32_t)std::min<int64_t>(c, k + K), T.nslots, job});
                T.nslots++;
            }
        }
    }
    T.split_begin.push_back(T.nslots);
}

// Heaviest items first (they are the tail otherwise); equal weights keep
// their order.  A stable LSD radix sort on (largest weight - weight), 8 bits a
// pass and only as many passes as the largest weight needs: the order
// std::stable_sort gives, in linear time (the plan of a 10^4^2 raster sorts
// about 13,000 items while the GPU waits).
void sort_items(std::vector<Item>& items) {
    const size_t n = items.size();
    if (n < 2) return;
    uint32_t wmax = 0;
    for (const Item& it : items) wmax = std::max<uint32_t>(wmax, (uint32_t)(it.k1 - it.k0));
    std::vector<Item> tmp(n);
    Item *src = items.data(), *dst = tmp.data();
    bool in_tmp = false;
    for (int shift = 0; shift < 32 && (wmax >> shift) != 0; shift += 8) {
        size_t cnt[257] = {};
        for (size_t i = 0; i < n; i++) cnt[((wmax - (uint32_t)(src[i].k1 - src[i].k0)) >> shift & 0xffu) + 1]++;
        for (int d = 0; d < 256; d++) cnt[d + 1] += cnt[d];
        for (size_t i = 0; i < n; i++) dst[cnt[(wmax - (uint32_t)(src[i].k1 - src[i].k0)) >> shift & 0xffu]++] = src[i];
        std::swap(src, dst);
        in_tmp = !in_tmp;
    }
    if (in_tmp) items.swap(tmp);
}

}  // namespace

// A planned density launch: work items and split tables written to the
// context's mapped staging (copied to device memory ahead of each launch),
// scratch allocated, kernels not yet launched.
struct mgk_dplan {
    const mgk_index* idx = nullptr;
    bool fp64 = false, count = false;
    DParams P{};
    TilePlan T;
    const int32_t *d_sb = nullptr, *d_sbeg = nullptr;
    unsigned long long *h_err = nullptr, *d_err = nullptr;
    size_t b_scr = 0;
    // device copy of the work list and split tables, refreshed from the
    // staging ahead of each launch
    void* d_tab = nullptr;
    const void* src_tab = nullptr;
    size_t b_tab = 0;
    bool staged = false;  // d_tab already filled (mgk_density_stage) for the next launch
};

static void dplan_release(mgk_ctx* ctx, mgk_dplan* D) {
    if (!D) return;
    if (D->T.nslots) mgk_free(ctx, D->P.scratch, D->b_scr);
    if (D->d_tab) mgk_free(ctx, D->d_tab, D->b_tab);
    delete D;
}

// n16 16-byte words from the mapped staging to device memory.
__global__ void k_stage_copy(uint4* __restrict__ dst, const uint4* src, size_t n16) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n16; i += (size_t)gridDim.x * blockDim.x)
        dst[i] = src[i];
}

// The kernels read the work list and split tables from device memory: a
// copy kernel moves them there from the mapped staging ahead of each launch,
// on the launch's stream.  Read in place, each CTA's item would cross the
// bus on its own, slowly while bulk copies (masks in, densities out) load it.
static int stage_tables(mgk_ctx* ctx, const mgk_dplan* D, cudaStream_t s) {
    if (!D->d_tab) return MGK_OK;
    const size_t n16 = D->b_tab / 16;
    const unsigned grid = (unsigned)std::max<size_t>(1, std::min<size_t>((size_t)ctx->sm_count, (n16 + 255) / 256));
    k_stage_copy<<<grid, 256, 0, s>>>(reinterpret_cast<uint4*>(D->d_tab), reinterpret_cast<const uint4*>(D->src_tab),
                                      n16);
    const cudaError_t ce = cudaGetLastError();
    if (ce != cudaSuccess) return mgk_cuda_fail(ctx, ce, "density work list");
    MGK_COUNT_LAUNCH(ctx, 1);
    return MGK_OK;
}

void mgk_density_discard(mgk_ctx* ctx, mgk_dplan* D) { dplan_release(ctx, D); }

// The counting kernel of a tile into staging slot `slot` (counts at offset 0).
static int counts_launch(mgk_ctx* ctx, const mgk_index* idx, const mgk_grid* g, int64_t row0, int64_t col0,
                         int64_t nr, int64_t nc, int slot, cudaStream_t s, bool zero_err) {
    if (nr <= 0 || nc <= 0) return MGK_OK;
    DParams P;
    fill_params(P, idx, g, row0, col0, nr, nc, nullptr, nullptr);
    P.err = zero_err ? ctx->d_counter + 7 : nullptr;  // other tiles' kernels may share the flag
    const int nbx_t = (int)((nc + kBC - 1) / kBC), nby_t = (int)((nr + kBR - 1) / kBR);
    const int nblk = nbx_t * nby_t;
    char *h_st = nullptr, *d_st = nullptr;
    const int st = mgk_host_stage_slot(ctx, slot, sizeof(int64_t) * nblk, (void**)&h_st, (void**)&d_st);
    if (st) return st;
    k_block_counts<<<(nblk + 255) / 256, 256, 0, s>>>(P, nbx_t, nby_t, reinterpret_cast<int64_t*>(d_st));
    const cudaError_t ce = cudaGetLastError();
    if (ce != cudaSuccess) return mgk_cuda_fail(ctx, ce, "density plan");
    MGK_COUNT_LAUNCH(ctx, 1);
    return MGK_OK;
}

// The plan of a tile from the counts in staging slot `slot` (its counting
// kernel has finished); the work list, split tables and error flag go into
// the same slot.
static int plan_from_counts(mgk_ctx* ctx, const mgk_index* idx, const mgk_grid* g, int64_t row0, int64_t col0,
                            int64_t nr, int64_t nc, const int64_t* counts, const float* d_mask, float* d_out,
                            unsigned long long* d_evals, bool fp64, int slot, mgk_dplan** out);

static int plan_counted(mgk_ctx* ctx, const mgk_index* idx, const mgk_grid* g, int64_t row0, int64_t col0,
                        int64_t nr, int64_t nc, const float* d_mask, float* d_out, unsigned long long* d_evals,
                        bool fp64, int slot, mgk_dplan** out) {
    *out = nullptr;
    if (nr <= 0 || nc <= 0) return MGK_OK;
    const int nbx_t = (int)((nc + kBC - 1) / kBC), nby_t = (int)((nr + kBR - 1) / kBR);
    char *h_st = nullptr, *d_st = nullptr;
    const int st = mgk_host_stage_slot(ctx, slot, sizeof(int64_t) * nbx_t * nby_t, (void**)&h_st, (void**)&d_st);
    if (st) return st;
    // the counts are consumed (plan_tile) before the slot is written again
    return plan_from_counts(ctx, idx, g, row0, col0, nr, nc, reinterpret_cast<const int64_t*>(h_st), d_mask, d_out,
                            d_evals, fp64, slot, out);
}

// The plan of a tile from its per-block candidate counts (host memory); the
// work list, split tables and error flag go into staging slot `slot`.
static int plan_from_counts(mgk_ctx* ctx, const mgk_index* idx, const mgk_grid* g, int64_t row0, int64_t col0,
                            int64_t nr, int64_t nc, const int64_t* counts, const float* d_mask, float* d_out,
                            unsigned long long* d_evals, bool fp64, int slot, mgk_dplan** out) {
    *out = nullptr;
    if (nr <= 0 || nc <= 0) return MGK_OK;
    mgk_dplan* D = new (std::nothrow) mgk_dplan();
    if (!D) return mgk_fail(ctx, MGK_ERR_INVALID, "density plan: out of host memory");
    D->idx = idx;
    D->fp64 = fp64;
    D->count = d_evals != nullptr;
    DParams& P = D->P;
    fill_params(P, idx, g, row0, col0, nr, nc, d_mask, d_out);
    P.evals = d_evals;
    P.err = ctx->d_counter + 7;
    const int nbx_t = (int)((nc + kBC - 1) / kBC), nby_t = (int)((nr + kBR - 1) / kBR);
    int st;
    TilePlan& T = D->T;
    plan_tile(counts, nbx_t, nby_t, ctx->sm_count, ctx->split_waves, 0, T);
    sort_items(T.items);
    const int32_t nslots = T.nslots;
    D->b_scr = sizeof(double) * (size_t)kCells * (size_t)std::max(nslots, 1);
    if (nslots && (st = mgk_alloc(ctx, (void**)&P.scratch, D->b_scr))) {
        delete D;
        return st;
    }
    // the work list, the split tables and the error flag in the staging:
    // [items | split blocks | split begins | err]
    auto up16 = [](size_t b) { return (b + 15) & ~(size_t)15; };
    const size_t b_items = sizeof(Item) * T.items.size();
    const size_t b_sb = sizeof(int32_t) * T.split_blocks.size(), b_sbeg = sizeof(int32_t) * T.split_begin.size();
    const size_t o_sb = up16(b_items), o_sbeg = o_sb + up16(b_sb), o_err = o_sbeg + up16(b_sbeg);
    char *h_st = nullptr, *d_st = nullptr;
    if ((st = mgk_host_stage_slot(ctx, slot, o_err + sizeof(unsigned long long), (void**)&h_st, (void**)&d_st))) {
        dplan_release(ctx, D);
        return st;
    }
    memcpy(h_st, T.items.data(), b_items);
    if (nslots) {
        memcpy(h_st + o_sb, T.split_blocks.data(), b_sb);
        memcpy(h_st + o_sbeg, T.split_begin.data(), b_sbeg);
    }
    D->b_tab = o_err;  // items and split tables (a 16-byte multiple)
    if ((st = mgk_alloc(ctx, &D->d_tab, D->b_tab))) {
        D->d_tab = nullptr;
        dplan_release(ctx, D);
        return st;
    }
    D->src_tab = d_st;
    const char* d_tab = static_cast<const char*>(D->d_tab);
    P.items = reinterpret_cast<const Item*>(d_tab);
    D->d_sb = reinterpret_cast<const int32_t*>(d_tab + o_sb);
    D->d_sbeg = reinterpret_cast<const int32_t*>(d_tab + o_sbeg);
    D->h_err = reinterpret_cast<unsigned long long*>(h_st + o_err);
    D->d_err = reinterpret_cast<unsigned long long*>(d_st + o_err);
    *D->h_err = 0;
    *out = D;
    return MGK_OK;
}

int mgk_density_prepare(mgk_ctx* ctx, const mgk_index* idx, const mgk_grid* g, int64_t row0, int64_t col0,
                        int64_t nr, int64_t nc, const float* d_mask, float* d_out, unsigned long long* d_evals,
                        bool fp64, mgk_dplan** out) {
    *out = nullptr;
    if (nr <= 0 || nc <= 0) return MGK_OK;
    int st = counts_launch(ctx, idx, g, row0, col0, nr, nc, 0, ctx->stream, true);
    if (st) return st;
    const cudaError_t ce = cudaStreamSynchronize(ctx->stream);
    if (ce != cudaSuccess) return mgk_cuda_fail(ctx, ce, "density plan");
    return plan_counted(ctx, idx, g, row0, col0, nr, nc, d_mask, d_out, d_evals, fp64, 0, out);
}

int mgk_density_counts_launch(mgk_ctx* ctx, const mgk_index* idx, const mgk_grid* g, int64_t row0, int64_t col0,
                              int64_t nr, int64_t nc, int slot, cudaStream_t s) {
    return counts_launch(ctx, idx, g, row0, col0, nr, nc, slot, s, false);
}

int mgk_density_plan_counted(mgk_ctx* ctx, const mgk_index* idx, const mgk_grid* g, int64_t row0, int64_t col0,
                             int64_t nr, int64_t nc, const float* d_mask, float* d_out, unsigned long long* d_evals,
                             int slot, mgk_dplan** out) {
    return plan_counted(ctx, idx, g, row0, col0, nr, nc, d_mask, d_out, d_evals, false, slot, out);
}

int mgk_density_plan_from_counts(mgk_ctx* ctx, const mgk_index* idx, const mgk_grid* g, int64_t row0, int64_t col0,
                                 int64_t nr, int64_t nc, const int64_t* counts, const float* d_mask, float* d_out,
                                 unsigned long long* d_evals, int slot, mgk_dplan** out) {
    return plan_from_counts(ctx, idx, g, row0, col0, nr, nc, counts, d_mask, d_out, d_evals, false, slot, out);
}

const int64_t* mgk_density_counts_host(mgk_ctx* ctx, int slot) {
    return static_cast<const int64_t*>(ctx->h_stage[slot]);
}

void mgk_density_set_tail_flag(mgk_dplan* D, unsigned* flag) {
    if (D) D->P.tail_flag = flag;
}

void mgk_density_set_mask_bits(mgk_dplan* D, const unsigned char* bits, int64_t stride) {
    if (!D) return;
    D->P.mask = nullptr;
    D->P.mbits = bits;
    D->P.mbstride = stride;
}

int mgk_density_stage(mgk_ctx* ctx, mgk_dplan* D, cudaStream_t s) {
    if (!D) return MGK_OK;
    const int st = stage_tables(ctx, D, s);
    if (st == MGK_OK) D->staged = true;
    return st;
}

int mgk_density_launch_plan(mgk_ctx* ctx, mgk_dplan* D, cudaStream_t s) {
    if (!D) return MGK_OK;
    const DParams& P = D->P;
    const bool varh = D->idx->varh;
    const unsigned grid = (unsigned)D->T.items.size();
    const int st = D->staged ? MGK_OK : stage_tables(ctx, D, s);
    if (st) return st;
    if (D->count) {
        if (varh) launch_density<true, true>(grid, s, P);
        else launch_density<false, true>(grid, s, P);
    } else {
        if (varh) launch_density<true, false>(grid, s, P);
        else launch_density<false, false>(grid, s, P);
    }
    MGK_COUNT_LAUNCH(ctx, 1);
    if (D->T.nslots) {
        k_merge<<<dim3((unsigned)D->T.split_blocks.size(), kMergeParts), 256, 0, s>>>(P, D->d_sb, D->d_sbeg);
        MGK_COUNT_LAUNCH(ctx, 1);
    }
    const cudaError_t ce = cudaGetLastError();
    if (ce != cudaSuccess) return mgk_cuda_fail(ctx, ce, "density");
    return MGK_OK;
}

int mgk_density_launch_split(mgk_ctx* ctx, mgk_dplan* D, cudaStream_t s, cudaStream_t s_merge, cudaEvent_t ev,
                             bool* merged_on_s_merge) {
    *merged_on_s_merge = false;
    if (!D) return MGK_OK;
    if (!D->T.nslots || !s_merge) return mgk_density_launch_plan(ctx, D, s);
    const DParams& P = D->P;
    const bool varh = D->idx->varh;
    const unsigned grid = (unsigned)D->T.items.size();
    int st = D->staged ? MGK_OK : stage_tables(ctx, D, s);
    if (st) return st;
    if (D->count) {
        if (varh) launch_density<true, true>(grid, s, P);
        else launch_density<false, true>(grid, s, P);
    } else {
        if (varh) launch_density<true, false>(grid, s, P);
        else launch_density<false, false>(grid, s, P);
    }
    MGK_COUNT_LAUNCH(ctx, 1);
    cudaError_t ce = cudaGetLastError();
    if (ce == cudaSuccess) ce = cudaEventRecord(ev, s);
    if (ce == cudaSuccess) ce = cudaStreamWaitEvent(s_merge, ev, 0);
    if (ce == cudaSuccess) {
        k_merge<<<dim3((unsigned)D->T.split_blocks.size(), kMergeParts), 256, 0, s_merge>>>(P, D->d_sb, D->d_sbeg);
        ce = cudaGetLastError();
    }
    if (ce != cudaSuccess) return mgk_cuda_fail(ctx, ce, "density");
    MGK_COUNT_LAUNCH(ctx, 1);
    *merged_on_s_merge = true;
    return MGK_OK;
}

int mgk_density_execute(mgk_ctx* ctx, mgk_dplan* D) {
    if (!D) return MGK_OK;
    cudaStream_t s = ctx->stream;
    DParams& P = D->P;
    const mgk_index* idx = D->idx;
    cudaError_t ce = cudaSuccess;
    int rc = MGK_OK;
    do {
        const unsigned grid = (unsigned)D->T.items.size();
        if ((rc = stage_tables(ctx, D, s))) break;
        cudaEventRecord(ctx->ev_a, s);
        if (D->fp64) {
            if (idx->varh) k_density_fp64<true><<<grid, kThreads, 0, s>>>(P);
            else k_density_fp64<false><<<grid, kThreads, 0, s>>>(P);
        } else if (D->count) {
            if (idx->varh) launch_density<true, true>(grid, s, P);
            else launch_density<false, true>(grid, s, P);
        } else {
            if (idx->varh) launch_density<true, false>(grid, s, P);
            else launch_density<false, false>(grid, s, P);
        }
        cudaEventRecord(ctx->ev_b, s);
        if ((ce = cudaGetLastError()) != cudaSuccess) break;
        MGK_COUNT_LAUNCH(ctx, 1);  // density (the counting kernel counts itself)
        if (D->T.nslots) {
            k_merge<<<dim3((unsigned)D->T.split_blocks.size(), kMergeParts), 256, 0, s>>>(P, D->d_sb, D->d_sbeg);
            if ((ce = cudaGetLastError()) != cudaSuccess) break;
            MGK_COUNT_LAUNCH(ctx, 1);
        }
        k_store_flag<<<1, 1, 0, s>>>(P.err, D->d_err);
        if ((ce = cudaGetLastError()) != cudaSuccess) break;
        MGK_COUNT_LAUNCH(ctx, 1);
        // the work list and scratch are released below: wait for the kernels
        ce = cudaStreamSynchronize(s);
        if (ce == cudaSuccess) cudaEventElapsedTime(&ctx->last_density_ms, ctx->ev_a, ctx->ev_b);
    } while (0);
    if (ce != cudaSuccess) rc = mgk_cuda_fail(ctx, ce, "density");
    else if (*D->h_err) rc = mgk_fail(ctx, MGK_ERR_TIMEOUT, "density: a shared-memory staging wait timed out");
    dplan_release(ctx, D);
    return rc;
}

int mgk_launch_density(mgk_ctx* ctx, const mgk_index* idx, const mgk_grid* g, int64_t row0, int64_t col0,
                       int64_t nr, int64_t nc, const float* d_mask, float* d_out,
                       unsigned long long* d_evals, bool fp64) {
    mgk_dplan* D = nullptr;
    const int st = mgk_density_prepare(ctx, idx, g, row0, col0, nr, nc, d_mask, d_out, d_evals, fp64, &D);
    if (st) return st;
    return mgk_density_execute(ctx, D);
}

// Several tiles in one density launch (plus one merge launch): the tiles
// are planned independently (their items and split slots are exactly those
// of mgk_launch_density), their items concatenated and ordered heaviest
// first, and each item finds its tile's parameters through its job index.
// Jobs with per-point bandwidths and jobs with a fixed one go to two
// launches.  evals (optional, device) receives per-job counters.
int mgk_launch_density_jobs(mgk_ctx* ctx, int njobs, const mgk_tile_job* jobs, unsigned long long* d_evals) {
    if (njobs <= 0) return MGK_OK;
    cudaStream_t s = ctx->stream;
    std::vector<DParams> P(njobs);
    std::vector<int> nbx(njobs), nby(njobs), off(njobs + 1, 0);
    for (int j = 0; j < njobs; j++) {
        const mgk_tile_job& J = jobs[j];
        fill_params(P[j], J.index, &J.grid, J.row0, J.col0, J.nrows, J.ncols, J.d_mask, J.d_out);
        P[j].evals = d_evals ? d_evals + j : nullptr;
        P[j].err = ctx->d_counter + 7;
        nbx[j] = J.nrows > 0 && J.ncols > 0 ? (int)((J.ncols + kBC - 1) / kBC) : 0;
        nby[j] = J.nrows > 0 && J.ncols > 0 ? (int)((J.nrows + kBR - 1) / kBR) : 0;
        off[j + 1] = off[j] + nbx[j] * nby[j];
    }
    const int nblk_all = off[njobs];
    if (nblk_all == 0) return MGK_OK;
    int st;
    // Plan tables travel through the context's mapped page-locked staging
    // (mgk_host_stage): no copy engine, so they never queue behind large
    // copies that other streams have in flight.
    char *h_st = nullptr, *d_st = nullptr;
    if ((st = mgk_host_stage(ctx, sizeof(int64_t) * nblk_all, (void**)&h_st, (void**)&d_st))) return st;
    cudaError_t ce = cudaSuccess;
    for (int j = 0; j < njobs && ce == cudaSuccess; j++) {
        const int nb = nbx[j] * nby[j];
        if (nb)
            k_block_counts<<<(nb + 255) / 256, 256, 0, s>>>(P[j], nbx[j], nby[j],
                                                             reinterpret_cast<int64_t*>(d_st) + off[j]);
        ce = cudaGetLastError();
    }
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(s);
    if (ce != cudaSuccess) return mgk_cuda_fail(ctx, ce, "density jobs plan");
    MGK_COUNT_LAUNCH(ctx, njobs);
    // plan each job; items of both bandwidth kinds, merges, slot offsets
    std::vector<Item> items_fix, items_var;
    std::vector<int4> merges;
    int32_t nslots = 0;
    std::vector<int32_t> slot0(njobs, 0);
    {
        const int64_t* counts = reinterpret_cast<const int64_t*>(h_st);
        for (int j = 0; j < njobs; j++) {
            if (!nbx[j]) continue;
            TilePlan T;
            plan_tile(counts + off[j], nbx[j], nby[j], ctx->sm_count, ctx->split_waves, j, T);
            slot0[j] = nslots;
            for (size_t b = 0; b < T.split_blocks.size(); b++)
                merges.push_back(make_int4(j, T.split_blocks[b], T.split_begin[b], T.split_begin[b + 1]));
            nslots += T.nslots;
            std::vector<Item>& dst = jobs[j].index->varh ? items_var : items_fix;
            dst.insert(dst.end(), T.items.begin(), T.items.end());
        }
    }
    sort_items(items_fix);
    sort_items(items_var);
    const size_t b_scr = sizeof(double) * (size_t)kCells * (size_t)std::max(nslots, 1);
    double* d_scr = nullptr;
    if (nslots && (st = mgk_alloc(ctx, (void**)&d_scr, b_scr))) return st;
    for (int j = 0; j < njobs; j++)
        P[j].scratch = d_scr ? d_scr + (size_t)slot0[j] * kCells : nullptr;  // slots are job-local
    // staging: [job parameters | items (fixed h, then per-point h) | merges | err]
    auto up16 = [](size_t v) { return (v + 15) & ~(size_t)15; };
    const size_t nitems = items_fix.size() + items_var.size();
    const size_t o_items = up16(sizeof(DParams) * njobs);
    const size_t o_mg = o_items + up16(sizeof(Item) * std::max<size_t>(nitems, 1));
    const size_t o_err = o_mg + up16(sizeof(int4) * std::max<size_t>(merges.size(), 1));
    if ((st = mgk_host_stage(ctx, o_err + sizeof(unsigned long long), (void**)&h_st, (void**)&d_st))) {
        mgk_free(ctx, d_scr, b_scr);
        return st;
    }
    memcpy(h_st, P.data(), sizeof(DParams) * njobs);
    memcpy(h_st + o_items, items_fix.data(), sizeof(Item) * items_fix.size());
    memcpy(h_st + o_items + sizeof(Item) * items_fix.size(), items_var.data(), sizeof(Item) * items_var.size());
    if (!merges.empty()) memcpy(h_st + o_mg, merges.data(), sizeof(int4) * merges.size());
    volatile unsigned long long* h_err = reinterpret_cast<unsigned long long*>(h_st + o_err);
    *h_err = 0;
    // the job parameters, items and merges in device memory (stage_tables)
    mgk_dplan tabs;
    tabs.b_tab = o_err;
    tabs.src_tab = d_st;
    if ((st = mgk_alloc(ctx, &tabs.d_tab, tabs.b_tab))) {
        mgk_free(ctx, d_scr, b_scr);
        return st;
    }
    const char* d_tab = static_cast<const char*>(tabs.d_tab);
    const DParams* d_jobs = reinterpret_cast<const DParams*>(d_tab);
    const Item* d_items = reinterpret_cast<const Item*>(d_tab + o_items);
    const int4* d_mg = reinterpret_cast<const int4*>(d_tab + o_mg);
    do {
        if ((st = stage_tables(ctx, &tabs, s))) break;
        cudaEventRecord(ctx->ev_a, s);
        if (!items_fix.empty()) {
            if (d_evals) launch_density_jobs<false, true>((unsigned)items_fix.size(), s, d_jobs, d_items);
            else launch_density_jobs<false, false>((unsigned)items_fix.size(), s, d_jobs, d_items);
            MGK_COUNT_LAUNCH(ctx, 1);
        }
        if (!items_var.empty()) {
            const Item* iv = d_items + items_fix.size();
            if (d_evals) launch_density_jobs<true, true>((unsigned)items_var.size(), s, d_jobs, iv);
            else launch_density_jobs<true, false>((unsigned)items_var.size(), s, d_jobs, iv);
            MGK_COUNT_LAUNCH(ctx, 1);
        }
        cudaEventRecord(ctx->ev_b, s);
        if ((ce = cudaGetLastError()) != cudaSuccess) break;
        if (!merges.empty()) {
            k_merge_jobs<<<dim3((unsigned)merges.size(), kMergeParts), 256, 0, s>>>(d_jobs, d_mg);
            if ((ce = cudaGetLastError()) != cudaSuccess) break;
            MGK_COUNT_LAUNCH(ctx, 1);
        }
        k_store_flag<<<1, 1, 0, s>>>(ctx->d_counter + 7, reinterpret_cast<unsigned long long*>(d_st + o_err));
        if ((ce = cudaGetLastError()) != cudaSuccess) break;
        MGK_COUNT_LAUNCH(ctx, 1);
        // the staging and the scratch are released below: wait for the kernels
        ce = cudaStreamSynchronize(s);
        if (ce == cudaSuccess) cudaEventElapsedTime(&ctx->last_density_ms, ctx->ev_a, ctx->ev_b);
    } while (0);
    if (ce != cudaSuccess) st = mgk_cuda_fail(ctx, ce, "density jobs");
    else if (st == MGK_OK && *h_err) st = mgk_fail(ctx, MGK_ERR_TIMEOUT, "density: a shared-memory staging wait timed out");
    if (st != MGK_OK && ce == cudaSuccess) (void)cudaStreamSynchronize(s);  // nothing in flight reads the tables
    mgk_free(ctx, d_scr, b_scr);
    mgk_free(ctx, tabs.d_tab, tabs.b_tab);
    tabs.d_tab = nullptr;
    return st;
}

// ---------------------------------------------------------------------------
// Density of one tile without allocating anything.
//
// mgk_density_tile takes its scratch (the per-block candidate counts, the
// work-item list and the FP64 partial sums of blocks split across CTAs) from
// the context's device allocator.  Some callers cannot let a library allocate
// device memory at that point: an application that reserves the GPU's memory
// up front for its own allocator or arena, or a latency-critical loop that
// forbids cudaMalloc/cudaFree (which may synchronise the whole device) once it
// is running.  For them this variant keeps all scratch in one fixed
// file-scope device array, g_density_scratch (kNaScratchBytes, about 12.3 MiB),
// which every GPU that loads the library holds until the process exits, and
// its host-side plan in fixed static arrays.  Limits: a tile of at most 4096 x
// 4096 cells (64 x 32 blocks of 64 x 128) and at most kNaMaxSlots split work
// items (heavy blocks get larger work items instead).  Inputs (index, mask) and
// the output tile are the caller's as for mgk_density_tile.
namespace {

constexpr int kNaMaxBlocks = 2048;
constexpr int kNaMaxItems = 12288;
constexpr int kNaMaxSlots = 192;
constexpr size_t kNaSlotBytes = sizeof(double) * kCells;
constexpr size_t na_round(size_t v) { return (v + 255) / 256 * 256; }
constexpr size_t kNaOffCounts = 0;
constexpr size_t kNaOffItems = na_round(kNaOffCounts + sizeof(int64_t) * kNaMaxBlocks);
constexpr size_t kNaOffSplit = na_round(kNaOffItems + sizeof(Item) * kNaMaxItems);
constexpr size_t kNaOffSplitBegin = na_round(kNaOffSplit + sizeof(int32_t) * kNaMaxSlots);
constexpr size_t kNaOffSlots = na_round(kNaOffSplitBegin + sizeof(int32_t) * (kNaMaxSlots + 1));
constexpr size_t kNaScratchBytes = kNaOffSlots + kNaSlotBytes * kNaMaxSlots;

static __device__ __align__(256) unsigned char g_density_scratch[kNaScratchBytes];

constexpr int kNaMaxDevices = 64;
unsigned char* g_na_addr[kNaMaxDevices];  // device address of g_density_scratch, per device
std::mutex g_na_mu;                       // guards g_na_addr and the static host plan below
int64_t g_na_counts[kNaMaxBlocks];
Item g_na_items[kNaMaxItems];
int32_t g_na_split[kNaMaxSlots];
int32_t g_na_split_begin[kNaMaxSlots + 1];

// Makes `device` current for a scope and restores the caller's device after.
struct NaDeviceScope {
    int prev = -1;
    cudaError_t err = cudaSuccess;
    explicit NaDeviceScope(int device) {
        if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
        if (prev != device) err = cudaSetDevice(device);
    }
    ~NaDeviceScope() {
        int cur = -1;
        if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
    }
};

}  // namespace

extern "C" int mgk_density_tile_noalloc(mgk_ctx* ctx, const mgk_index* idx, const mgk_grid* g, int64_t row0,
                                        int64_t col0, int64_t nr, int64_t nc, const float* d_mask, float* d_out) {
    if (!ctx || !idx || !g || !d_out || !(g->cs > 0.0f) || g->ncols <= 0 || g->nrows <= 0)
        return mgk_fail(ctx, MGK_ERR_INVALID, "density_tile_noalloc: bad arguments");
    if (row0 < 0 || col0 < 0 || nr < 0 || nc < 0 || row0 + nr > g->nrows || col0 + nc > g->ncols)
        return mgk_fail(ctx, MGK_ERR_INVALID, "density_tile_noalloc: tile outside the raster");
    if (nr == 0 || nc == 0) return MGK_OK;
    const int nbx_t = (int)((nc + kBC - 1) / kBC), nby_t = (int)((nr + kBR - 1) / kBR);
    const int nblk = nbx_t * nby_t;
    if (nr > 4096 || nc > 4096 || nblk > kNaMaxBlocks)
        return mgk_fail(ctx, MGK_ERR_INVALID,
                        "density_tile_noalloc: tile of " + std::to_string(nr) + " x " + std::to_string(nc) +
                            " cells exceeds the fixed scratch (at most 4096 x 4096 cells)");
    std::lock_guard<std::mutex> lock(g_na_mu);
    if (ctx->device < 0 || ctx->device >= kNaMaxDevices)
        return mgk_fail(ctx, MGK_ERR_INVALID, "density_tile_noalloc: device index out of range");
    // the context's device stays current for the whole call (the address
    // look-up, the kernels and the copies); the caller's is restored on return
    NaDeviceScope scope(ctx->device);
    if (scope.err != cudaSuccess) return mgk_cuda_fail(ctx, scope.err, "density_tile_noalloc: cudaSetDevice");
    // set-up, once per device, with that device current: the host-side name of
    // a __device__ array is not its device address, so look the address up
    if (!g_na_addr[ctx->device]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_density_scratch);
        if (e != cudaSuccess) return mgk_cuda_fail(ctx, e, "cudaGetSymbolAddress(g_density_scratch)");
        g_na_addr[ctx->device] = static_cast<unsigned char*>(p);
    }
    unsigned char* base = g_na_addr[ctx->device];
    int64_t* d_counts = reinterpret_cast<int64_t*>(base + kNaOffCounts);
    Item* d_items = reinterpret_cast<Item*>(base + kNaOffItems);
    int32_t* d_sb = reinterpret_cast<int32_t*>(base + kNaOffSplit);
    int32_t* d_sbeg = reinterpret_cast<int32_t*>(base + kNaOffSplitBegin);
    cudaStream_t s = ctx->stream;

    DParams P;
    fill_params(P, idx, g, row0, col0, nr, nc, d_mask, d_out);
    P.evals = nullptr;
    P.err = ctx->d_counter + 7;
    P.scratch = reinterpret_cast<double*>(base + kNaOffSlots);

    // plan: candidates per block (device) -> work items (host, static arrays)
    // (k_block_counts also clears the staging-wait flag P.err of this launch)
    k_block_counts<<<(nblk + 255) / 256, 256, 0, s>>>(P, nbx_t, nby_t, d_counts);
    cudaError_t ce = cudaGetLastError();
    if (ce == cudaSuccess)
        ce = cudaMemcpyAsync(g_na_counts, d_counts, sizeof(int64_t) * nblk, cudaMemcpyDeviceToHost, s);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(s);
    if (ce != cudaSuccess) return mgk_cuda_fail(ctx, ce, "density_tile_noalloc plan");
    int64_t total = 0;
    for (int b = 0; b < nblk; b++) total += g_na_counts[b];
    const int64_t slots_resident = (int64_t)ctx->sm_count * MGK_DENSITY_MIN_CTAS;
    int64_t K = std::max<int64_t>(2048, total / std::max<int64_t>(1, slots_resident * ctx->split_waves));
    K = (K + kMB - 1) / kMB * kMB;
    for (;;) {  // grow the item size until the split items fit the fixed slots
        int64_t need = 0;
        for (int b = 0; b < nblk; b++)
            if (g_na_counts[b] > K) need += (g_na_counts[b] + K - 1) / K;
        if (need <= kNaMaxSlots) break;
        K *= 2;
    }
    int nitems = 0, nsplit = 0;
    int32_t nslots = 0;
    for (int b = 0; b < nblk; b++) {
        const int64_t c = g_na_counts[b];
        const int bxi = b % nbx_t, byi = b / nbx_t;
        if (c <= K) {
            g_na_items[nitems++] = {bxi, byi, 0, (int32_t)c, -1, 0};
        } else {
            g_na_split[nsplit] = b;
            g_na_split_begin[nsplit++] = nslots;
            for (int64_t k = 0; k < c; k += K)
                g_na_items[nitems++] = {bxi, byi, (int32_t)k, (int32_t)std::min<int64_t>(c, k + K), nslots++, 0};
        }
    }
    g_na_split_begin[nsplit] = nslots;
    // heaviest items first; ties keep block order (std::sort allocates nothing)
    for (int i = 0; i < nitems; i++) g_na_items[i].pad = i;
    std::sort(g_na_items, g_na_items + nitems, [](const Item& a, const Item& b) {
        const int32_t ca = a.k1 - a.k0, cb = b.k1 - b.k0;
        return ca != cb ? ca > cb : a.pad < b.pad;
    });
    ce = cudaMemcpyAsync(d_items, g_na_items, sizeof(Item) * nitems, cudaMemcpyHostToDevice, s);
    if (ce == cudaSuccess && nsplit) {
        ce = cudaMemcpyAsync(d_sb, g_na_split, sizeof(int32_t) * nsplit, cudaMemcpyHostToDevice, s);
        if (ce == cudaSuccess)
            ce = cudaMemcpyAsync(d_sbeg, g_na_split_begin, sizeof(int32_t) * (nsplit + 1), cudaMemcpyHostToDevice, s);
    }
    if (ce != cudaSuccess) return mgk_cuda_fail(ctx, ce, "density_tile_noalloc upload");
    P.items = d_items;
    if (idx->varh) launch_density<true, false>((unsigned)nitems, s, P);
    else launch_density<false, false>((unsigned)nitems, s, P);
    if ((ce = cudaGetLastError()) != cudaSuccess) return mgk_cuda_fail(ctx, ce, "density_tile_noalloc");
    MGK_COUNT_LAUNCH(ctx, 2);
    if (nsplit) {
        k_merge<<<dim3((unsigned)nsplit, kMergeParts), 256, 0, s>>>(P, d_sb, d_sbeg);
        if ((ce = cudaGetLastError()) != cudaSuccess) return mgk_cuda_fail(ctx, ce, "density_tile_noalloc merge");
        MGK_COUNT_LAUNCH(ctx, 1);
    }
    // the static host plan is reused by the next call: finish this one first
    unsigned long long err = 0;
    ce = cudaMemcpyAsync(&err, P.err, sizeof(err), cudaMemcpyDeviceToHost, s);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(s);
    if (ce != cudaSuccess) return mgk_cuda_fail(ctx, ce, "density_tile_noalloc");
    if (err) return mgk_fail(ctx, MGK_ERR_TIMEOUT, "density_tile_noalloc: a shared-memory staging wait timed out");
    return MGK_OK;
}
