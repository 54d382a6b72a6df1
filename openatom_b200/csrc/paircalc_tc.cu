// PairCalculator products on the tcgen05 tensor cores (mixed precision).
//
// The same two products as the SIMT path (ckPairCalculator.C multiplyForward
// and bwMultiplyHelper; see paircalc.cu), written as split-BF16 compensated
// products.  Every FP64 operand element is rounded to FP32 and split exactly
// into three BF16 levels, f = h + m + l, and
//
//     a b ~ l_a h_b + h_a l_b + m_a m_b + m_a h_b + h_a m_b + h_a h_b
//
// (the level pairs of total order <= 2; the dropped ones are O(2^-24 |ab|)) is
// accumulated by tcgen05.mma (kind::f16, BF16 in, FP32 accumulators in TMEM),
// smallest terms first, h_a h_b in an accumulator of its own.  That one holds
// at most 128 reals of K: it is then read back
// (tcgen05.ld) and added into an FP64 copy of the tile kept in the other half
// of TMEM (two 32-bit columns per element, read and written back with
// tcgen05.ld / tcgen05.st).  The five
// small products (2^-7 of the total) run over the CTA's whole K range in FP32
// and join the FP64 tile in the epilogue: their rounding stays well below the
// hi*hi groups' own.  The sums over the groups, the split-K slabs and the
// epilogue terms are FP64.
//
// One CTA = one 128 x 128 output tile (M = N = 128 MMA) and one K range,
// one CTA per SM, 17 warps in two roles:
//   * warps 0-15 (workers) bring the FP64 operand chunks (KC reals) into NST
//     shared-memory stages with cp.async, split a stage into BF16 levels in
//     the K-major no-swizzle core-matrix layout (8 rows x 16 bytes per core
//     matrix; the two 8-element K halves of a 16-wide K step 128 bytes apart,
//     8-row groups 256 bytes apart; per K step the three levels 4 KB apart),
//     applying the per-point weight (a power of two: exact) on the way, and
//     after every 128 reals fold the hi*hi accumulator into the FP64 tile,
//     releasing it to the MMA warp as soon as it is read;
//   * warp 16 issues the 6 MMAs per K step into two FP32 TMEM accumulators
//     (the five small products in columns 0-127, hi*hi in columns 128-255;
//     the FP64 tile holds columns 256-511), commits them to an mbarrier, and
//     keeps the stages of a pre-split operand filled.
// An operand that many CTAs share (T in the back-multiply) is split once, by
// k_presplit, into its BF16 levels
// in global memory in the same core-matrix image; the MMA warp brings its
// chunks in with bulk copies (cp.async.bulk, one per chunk) and only the
// other operand is split in the CTA.
//
// Handshakes (all mbarriers): full[b] (workers' chunk in split buffer b),
// done[b] (MMAs of the chunk that used buffer b completed), tfree (hi*hi
// accumulator read back), pfull[s] (pre-split stage s landed).  Every wait is
// bounded (1 s) and also ends when the other role has raised `stop`; the CTA
// then records an error bit in *err, drains its copies, waits (bounded) for
// its MMAs, releases TMEM and returns without writing its tile.
//
//   overlap   (MODE 0): part[ks](i,j) = sum_{k in slab ks} w(k) A[i][k] B[j][k]
//   backmul   (MODE 1): out[i][p] = alpha w(p) (sum_{j != i} M(j,i) in[j][p]
//                                   + M(i,i) in[i][p]) + beta out[i][p]
// The backmul takes the diagonal of M out of the tensor-core product and adds
// it in FP64 in the epilogue (psi.T with T near I is then accurate relative
// to T - diag T); the overlap of one operand with itself (S) sums its
// diagonal in FP64 from the FP64 stage.
//
// The EES products (cp_ees_nonlocal.C's Z sums and psi force, evaluated in G
// space) follow at the end of the file: both of their operands are split once
// in global memory into two FP16 levels of power-of-two scaled values,
// x s = h + m (22 significant bits of the FP32 value; s brings the largest
// magnitude to [2^13, 2^14)), and multiplied as h m + m h + h h (three MMAs
// per K step, kind::f16 with FP16 A and B); k_pp_tc (the sums, split-K with
// FP64 folds every 512 reals) and k_pf_tc (the psi force of both atom types,
// persistent over point tiles) stream both operands with bulk copies and
// leave the CTA no operand work.
//
// Which kernel runs a PairCalc product (mixed context):
//   overlap S, lambda     fewer than 256 states: k_pc_tc MODE 0 (in-CTA split);
//                         256 or more: both operands split once into BF16
//                         levels (k_presplit) and streamed by k_pp_tc<3,false>
//   back-multiply         nin <= 128: k_bm_tc (two CTAs per SM, PsiV reset in
//                         the epilogue); 128 < nin < 256: k_pc_tc MODE 1;
//                         256 or more: in^T split by k_presplit_t and streamed
//                         by k_pp_tc<3,true>
#include "ctx.cuh"
#include "tc_sm100.cuh"

namespace pctc {

constexpr int ROWS = 128;                 // tile rows of A (M) and of B (N)
constexpr int NLV = 3;                    // BF16 levels per element (PairCalc products)
constexpr int NLV_H = 2;                  // FP16 levels per element (EES products)
constexpr int TILE_B = ROWS * 16 * 2;     // one K step, one level, one operand: 4 KB
constexpr int STEP_B = NLV * TILE_B;      // one K step, all levels: 12 KB
constexpr int STEP_H = NLV_H * TILE_B;    // the same, FP16 levels: 8 KB
constexpr int NW = 512;                   // worker threads (warps 0-15)
constexpr int MMA_WARP = NW / 32;         // warp 16 issues the MMAs
constexpr int NTHR = NW + 32;
constexpr int NSTP_MAX = 5;               // shared-memory stages of a pre-split operand (at most)
constexpr int WBAR = 1;                   // named barrier of the workers
constexpr uint32_t IDESC = tc::idesc_bf16_f32(ROWS, ROWS);
constexpr uint32_t IDESC_H = tc::idesc_f16_f32(ROWS, ROWS);
constexpr uint32_t TMEM_COLS = 512;       // two FP32 accumulators + the FP64 tile
constexpr uint32_t TMEM_F64 = 2 * ROWS;   // first column of the FP64 tile

template <int MODE, int NLD, int NST, int KC>
struct Cfg {
  static constexpr int KS = KC / 16;                     // MMA K steps per chunk
  static constexpr int U = KC / 8;                       // 8-element units per row
  // chunks per TMEM group: the hi*hi accumulator holds 128 reals of K (S
  // must stay orthonormal to 1e-8)
  static constexpr int NF = 128 / KC;
  static constexpr int RS = KC + 2;                      // row stride of a [128][KC] FP64 stage
  static constexpr int RSP = ROWS + 2;                   // row stride of a [KC][128] FP64 stage
  static constexpr int STEP = STEP_B;                    // one K step, all levels
  static constexpr int OPB = KS * STEP;                  // one operand of one chunk, split
  // operands split in the CTA (CA, CB) or pre-split in global memory (PB)
  static constexpr bool CA = true, CB = MODE == 0;
  static constexpr bool PA = false, PB = MODE == 1;
  static constexpr bool PRE = PA || PB;
  // pre-split stages: as deep as shared memory allows (the back-multiply's
  // FP64 [KC][128] stages leave room for 3)
  static constexpr int NSTP = MODE == 1 ? 3 : NSTP_MAX;
  static constexpr int NCONV = (CA ? 1 : 0) + (CB ? 1 : 0);
  static constexpr int RAW0 = ROWS * RS * 8;             // [128][KC] FP64
  static constexpr int WOFF = RAW0 * NLD;                // MODE 0: point weights after the rows
  // one stage: MODE 0 the FP64 rows; MODE 1 in[j][p]
  static constexpr int RAW = MODE == 0 ? WOFF + KC / 2 * 8 : KC * RSP * 8;
  static constexpr int CONV = 2 * NCONV * OPB;           // split operands, two chunk buffers
  static constexpr int PREB = PRE ? NSTP * OPB : 0;      // pre-split operand stages
  static constexpr int BYTES = 1024 + CONV + PREB + NST * RAW;  // + alignment slack
  static_assert(KC % 16 == 0 && 128 % KC == 0, "chunk");
  static_assert(RAW % 16 == 0 && OPB % 1024 == 0, "stage alignment");
  static_assert(ROWS * U * (MODE == 0 ? NLD : 1) == NW, "one 8-element unit per worker");
  static_assert(ROWS * (KC / 2) % NW == 0 && KC * (ROWS / 2) % NW == 0, "copy mapping");
};

struct Args {
  // overlap: A [M][lda], B [N][ldb] (K reals per row), w per complex point
  // backmul: A = in [nin][lda], B = Mcm (column i at Mcm + i ldb), w per point
  const double* A;
  const double* B;
  const double* w;
  int lda, ldb;
  int M, N, K;       // overlap: tile extents and reals; backmul: M = K points (reals), N = nout
  int nin;           // backmul inner dimension
  int kslab;         // overlap K slab per split
  int same;          // overlap: A and B are the same matrix (S)
  double* part;      // overlap partial tiles [nsplit][N][M] (column-major, ld = M)
  double* out;       // backmul output [nout][ldo]
  int ldo;
  double alpha, beta;
  // pre-split operand (MODE 1: B = M^T without its diagonal): [row tile][K
  // step][level][4 KB], pre_nsp K steps per row tile
  const uint8_t* pre;
  int pre_nsp;
  int* err;
};

// byte offset of (row r, k) in one K-step tile (k < 16), and the FP16
// two-level split of 8 scaled values of a row (tc_sm100.cuh)
using tc::core_off;
using tc::split_store_h;
static_assert(tc::CM_TILE == TILE_B, "core-matrix tile");

// 8 FP32 values of one row (8 consecutive K) -> three BF16 levels, stored as
// 16 bytes at dst + v TILE_B
__device__ __forceinline__ void split_store(uint8_t* dst, const float (&f)[8]) {
  uint32_t lv[NLV][4];
#pragma unroll
  for (int e = 0; e < 4; ++e) tc::split3_pair(f[2 * e], f[2 * e + 1], lv[0][e], lv[1][e], lv[2][e]);
#pragma unroll
  for (int v = 0; v < NLV; ++v)
    *reinterpret_cast<uint4*>(dst + v * TILE_B) = make_uint4(lv[v][0], lv[v][1], lv[v][2], lv[v][3]);
}

// FP64 values rounded to FP32 and scaled by their point's weight (a power of
// two, so the levels of the product are the weighted levels exactly)
__device__ __forceinline__ void to_f32(const double (&x)[8], const float (&ws)[4], float (&f)[8]) {
#pragma unroll
  for (int e = 0; e < 8; ++e) f[e] = (float)x[e] * ws[e >> 1];
}

struct PreArgs {
  const double* src;  // element (row, k) at src[row ldr + k]; ldr even, src 16-byte aligned
  long long ldr;
  int rows, K, nsp;   // nsp K steps (16 reals) per row tile, 16 nsp >= K, zero past K
  const double* w;    // weight per complex point k / 2 (a power of two), or none
  int zero_diag;      // element (i, i) taken as zero
  uint8_t* dst;       // [row tile][step][level][4 KB]
  uint8_t* dst2;      // the unweighted levels as well (the B operand of S), or none
};

// One warp = 16 rows x 16 reals of one K step and row tile: lane -> row
// (lane & 7) + 8 (lane >> 4) of the warp's pair of 8-row groups, K half
// (lane >> 3) & 1, so that each level's 512 bytes are written contiguously.
__global__ void __launch_bounds__(256) k_presplit(const PreArgs a) {
  const long long wid = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  const long long nwarps = (long long)cdiv(a.rows, ROWS) * a.nsp * 8;
  if (wid >= nwarps) return;
  const int gp = (int)(wid % 8);
  const long long rest = wid / 8;
  const int s = (int)(rest % a.nsp);
  const long long rt = rest / a.nsp;
  const int rl = (lane & 7) + 8 * (lane >> 4) + 16 * gp;
  const int kh = (lane >> 3) & 1;
  const long long row = rt * ROWS + rl;
  const int k0 = 16 * s + 8 * kh;
  double x[8];
#pragma unroll
  for (int e = 0; e < 8; ++e) x[e] = 0.0;
  if (row < a.rows) {
    const double* g = a.src + row * a.ldr + k0;
#pragma unroll
    for (int e = 0; e < 8; e += 2) {
      if (k0 + e + 1 < a.K) {
        const double2 v = *reinterpret_cast<const double2*>(g + e);
        x[e] = v.x;
        x[e + 1] = v.y;
      } else if (k0 + e < a.K) {  // odd K: the row's last element
        x[e] = g[e];
      }
    }
    if (a.zero_diag) {
#pragma unroll
      for (int e = 0; e < 8; ++e)
        if (k0 + e == row) x[e] = 0.0;
    }
  }
  float ws[4] = {1.f, 1.f, 1.f, 1.f};
  if (a.w) {
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      const int pt = (k0 >> 1) + e;
      if (2 * pt < a.K) ws[e] = (float)a.w[pt];
    }
  }
  float f[8];
  const size_t off = ((size_t)rt * a.nsp + s) * STEP_B + core_off(rl, 8 * kh);
  if (a.dst2) {
    const float one[4] = {1.f, 1.f, 1.f, 1.f};
    to_f32(x, one, f);
    split_store(a.dst2 + off, f);
  }
  to_f32(x, ws, f);
  split_store(a.dst + off, f);
}

template <int MODE, int NLD, int NST, int KC>
__global__ void __launch_bounds__(NTHR, 1) k_pc_tc(const Args p) {
  using C = Cfg<MODE, NLD, NST, KC>;
  constexpr int KS = C::KS, U = C::U, NF = C::NF, RS = C::RS, RSP = C::RSP;
  constexpr bool DIAG = MODE == 0;
  extern __shared__ uint8_t dsm[];
  constexpr int NSTP = C::NSTP;
  __shared__ uint64_t full[2], done[2], tfree, pfull[NSTP];
  __shared__ uint32_t tslot;
  __shared__ int stop_s, issued_s;
  __shared__ double diag_s[DIAG ? ROWS : 1];
  volatile int* stop = &stop_s;
  const uint32_t s0 = tc::smem_u32(dsm);
  uint8_t* base = dsm + (((s0 + 1023u) & ~1023u) - s0);
  const uint32_t bf_s = tc::smem_u32(base);  // split buffers [2][NCONV][KS][level][4 KB]
  uint8_t* pre_base = base + C::CONV;        // pre-split stages [NSTP][KS][level][4 KB]
  double* raw = reinterpret_cast<double*>(base + C::CONV + C::PREB);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

  int r0, c0, kbeg, kend;
  if (MODE == 0) {
    r0 = blockIdx.x * ROWS;
    c0 = blockIdx.y * ROWS;
    kbeg = blockIdx.z * p.kslab;
    kend = min(p.K, kbeg + p.kslab);
  } else {
    r0 = blockIdx.x * ROWS;   // points
    c0 = blockIdx.y * ROWS;   // output states
    kbeg = 0;
    kend = p.nin;
  }
  const int nch = kend > kbeg ? (kend - kbeg + KC - 1) / KC : 0;
  // S (A and B the same rows): its diagonal is summed in FP64 from the FP64
  // stage, and B's levels are A's without the weight
  const bool same = MODE == 0 && p.same && r0 == c0;

  if (warp == 0) tc::tmem_alloc(&tslot, TMEM_COLS);
  if (tid == 0) {
    for (int i = 0; i < 2; ++i) {
      tc::mbar_init(&full[i], NW / 32);  // one arrival per worker warp
      tc::mbar_init(&done[i], 1);
    }
    tc::mbar_init(&tfree, NW / 32);
    for (int i = 0; i < NSTP; ++i) tc::mbar_init(&pfull[i], 1);
    stop_s = 0;
    issued_s = 0;
    tc::fence_mbar_init();
  }
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tbase = tslot;

  // split buffer of chunk buffer `buf`, operand op (0 = A, 1 = B)
  auto conv_off = [](int buf, int op) -> int {
    return (buf * C::NCONV + ((op == 1 && C::CA) ? 1 : 0)) * C::OPB;
  };

  double dacc = 0.0;
  // a worker warp's slice of TMEM: lanes 32 (warp % 4).., tile columns 32 (warp / 4)..
  const uint32_t tlanes = (uint32_t)(32 * (warp & 3)) << 16;
  const uint32_t tf64 = tbase + tlanes + TMEM_F64 + (uint32_t)(64 * ((warp >> 2) & 3));

  if (warp == MMA_WARP) {
    // ---------------- MMA warp (lane 0 works, the warp stays converged)
    if (lane == 0) {
      int bad = 0, issued = 0, req = 0;
      const int prow = C::PA ? blockIdx.x : blockIdx.y;  // row tile of the pre-split operand
      auto pre_load = [&](int c) {
        const int st = c % NSTP;
        const uint8_t* src =
            p.pre + ((size_t)prow * p.pre_nsp + (size_t)((kbeg + c * KC) >> 4)) * C::STEP;
        tc::mbar_expect_tx(&pfull[st], C::OPB);
        tc::bulk_g2s(pre_base + (size_t)st * C::OPB, src, C::OPB, &pfull[st]);
      };
      // the MMAs of chunk ch, smallest level products first; the first chunk
      // of a group waits for the hi*hi accumulator's read-back (tfree) before
      // it overwrites it.  The commit covers whatever was issued.
      auto issue = [&](int ch) -> bool {
        const int buf = ch & 1, g = ch / NF;
        const bool first = ch % NF == 0;
        const uint32_t pre_s = bf_s + (uint32_t)(C::CONV + (ch % NSTP) * C::OPB);
        const uint32_t a0 = C::PA ? pre_s : bf_s + (uint32_t)conv_off(buf, 0);
        const uint32_t b0 = C::PB ? pre_s : bf_s + (uint32_t)conv_off(buf, 1);
        // level pairs, smallest first; the last (h h) goes to its own accumulator
        constexpr int LA[6] = {2, 0, 1, 1, 0, 0};
        constexpr int LB[6] = {0, 2, 1, 0, 1, 0};
        bool ok = true;
#pragma unroll
        for (int s = 0; s < KS; ++s) {
#pragma unroll
          for (int t = 0; t < 6; ++t) {
            const bool zero = first && s == 0 && (t == 5 || (t == 0 && ch == 0));
            if (first && s == 0 && t == 5 && g >= 1 && ok) {
              ok = tc::mbar_wait_or(&tfree, (g - 1) & 1, stop);
              tc::fence_after_sync();
            }
            const uint64_t da = tc::smem_desc_kmajor(a0 + s * C::STEP + LA[t] * TILE_B, 128, 256);
            const uint64_t db = tc::smem_desc_kmajor(b0 + s * C::STEP + LB[t] * TILE_B, 128, 256);
            if (ok) tc::mma_bf16(t == 5 ? tbase + ROWS : tbase, da, db, IDESC, zero ? 0u : 1u);
          }
        }
        tc::commit(&done[buf]);
        return ok;
      };
      if (C::PRE)
        for (; req < nch && req < NSTP; ++req) pre_load(req);
      for (int ch = 0; ch < nch; ++ch) {
        // chunk split, pre-split chunk landed
        if (!tc::mbar_wait_or(&full[ch & 1], (ch >> 1) & 1, stop)) {
          bad = 1;
          break;
        }
        if (C::PRE && !tc::mbar_wait_or(&pfull[ch % NSTP], (ch / NSTP) & 1, stop)) {
          bad = 1;
          break;
        }
        tc::fence_after_sync();
        const bool ok = issue(ch);
        issued = ch + 1;
        if (!ok) {
          bad = 1;
          break;
        }
        if (C::PRE && ch >= 1 && req < nch) {  // refill chunk ch - 1's stage with chunk req
          if (!tc::mbar_wait_or(&done[(ch - 1) & 1], ((ch - 1) >> 1) & 1, stop)) {
            bad = 1;
            break;
          }
          pre_load(req++);
        }
      }
      if (bad) {
        *stop = 1;
        for (int c = issued; c < req; ++c)  // requested copies land before the CTA exits
          tc::mbar_wait(&pfull[c % NSTP], (c / NSTP) & 1);
      }
      issued_s = issued;
    }
    __syncwarp();
  } else {
    // ---------------- workers
    // copies of chunk ch into stage st
    auto load = [&](int ch, int st) {
      const int k0 = kbeg + ch * KC;
      double* ra = raw + (size_t)st * (C::RAW / 8);
      if (MODE == 0) {
#pragma unroll
        for (int op = 0; op < NLD; ++op) {
          const double* src = op == 0 ? p.A : p.B;
          const int ld = op == 0 ? p.lda : p.ldb;
          const int rr0 = op == 0 ? r0 : c0, nr = op == 0 ? p.M : p.N;
          double* dst = ra + op * (C::RAW0 / 8);
          if (op == 0 && p.w && tid < KC / 4) {  // weights of points k0/2 .. (k0 + KC)/2
            const int pt = (k0 >> 1) + 2 * tid;
            const int nb = 2 * pt + 2 < kend ? 16 : (2 * pt < kend ? 8 : 0);
            tc::cp16(ra + C::WOFF / 8 + 2 * tid, nb ? p.w + pt : p.w, nb);
          }
#pragma unroll
          for (int it = 0; it < ROWS * (KC / 2) / NW; ++it) {
            const int q = tid + NW * it;
            const int r = q / (KC / 2), pc = q % (KC / 2);
            const int k = k0 + 2 * pc;
            const bool ok = rr0 + r < nr && k < kend;  // kend even: the pair is inside
            const double* g = ok ? src + (size_t)(rr0 + r) * ld + k : src;
            tc::cp16(dst + r * RS + 2 * pc, g, ok ? 16 : 0);
          }
        }
      } else {
        // in[j][p] rows j = k0 .. k0 + KC, 128 points from r0
#pragma unroll
        for (int it = 0; it < KC * (ROWS / 2) / NW; ++it) {
          const int q = tid + NW * it;
          const int jj = q / (ROWS / 2), pc = q % (ROWS / 2);
          const int j = k0 + jj, pt = r0 + 2 * pc;
          const bool ok = j < kend && pt < p.M;  // M (reals) even
          const double* g = ok ? p.A + (size_t)j * p.lda + pt : p.A;
          tc::cp16(ra + jj * RSP + 2 * pc, g, ok ? 16 : 0);
        }
      }
    };

    // stage st (chunk ch) -> split buffer buf: one 8-element unit per worker
    // (MODE 0 with two operands: A to workers < 256, B to the rest)
    auto convert = [&](int ch, int st, int buf) {
      const int k0 = kbeg + ch * KC;
      const double* ra = raw + (size_t)st * (C::RAW / 8);
      const int op = (MODE == 0 && NLD == 2) ? (tid >> 8) : 0;
      const int q = (MODE == 0 && NLD == 2) ? (tid & 255) : tid;
      const int r = (q & 7) + 8 * ((q >> 3) / U), u = (q >> 3) % U;
      const int off = (u >> 1) * C::STEP + core_off(r, (u & 1) * 8);
      uint8_t* dA = base + conv_off(buf, 0) + off;
      uint8_t* dB = base + conv_off(buf, 1) + off;
      const float one[4] = {1.f, 1.f, 1.f, 1.f};
      double x[8];
      float f[8];
      if (MODE == 1) {  // A[p][j] = in[j][p] from the [KC][128] stage
#pragma unroll
        for (int e = 0; e < 8; ++e) x[e] = ra[(8 * u + e) * RSP + r];
        to_f32(x, one, f);
        split_store(dA, f);
        return;
      }
      const double2* s2 =
          reinterpret_cast<const double2*>(ra + op * (C::RAW0 / 8) + r * RS + 8 * u);
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const double2 v = s2[e];
        x[2 * e] = v.x;
        x[2 * e + 1] = v.y;
      }
      if (op == 1) {
        to_f32(x, one, f);
        split_store(dB, f);
        return;
      }
      float ws[4] = {1.f, 1.f, 1.f, 1.f};
      if (p.w) {  // staged with the chunk (zero past the end, where x is zero too)
        const double2* w2 = reinterpret_cast<const double2*>(ra + C::WOFF / 8 + 4 * u);
        const double2 wa = w2[0], wb = w2[1];
        ws[0] = (float)wa.x;
        ws[1] = (float)wa.y;
        ws[2] = (float)wb.x;
        ws[3] = (float)wb.y;
      }
      if (same) {
        double d = 0.0;
#pragma unroll
        for (int e = 0; e < 8; ++e) d = fma((double)ws[e >> 1] * x[e], x[e], d);
        dacc += d;
      }
      if (NLD == 1) {
        to_f32(x, one, f);
        split_store(dB, f);
      }
      to_f32(x, ws, f);
      split_store(dA, f);
    };

    // group of chunk c (its last), once its MMAs are done: the hi*hi
    // accumulator is read, released to the MMA warp and added into the FP64
    // tile (the first group's is stored), 8 columns at a time
    auto flush = [&](int c) -> bool {
      const int g = c / NF;
      if (!__all_sync(0xffffffffu, tc::mbar_wait_or(&done[c & 1], (c >> 1) & 1, stop)))
        return false;
      tc::fence_after_sync();
      float v[32];
      tc::tmem_ld32(tbase + tlanes + (uint32_t)(ROWS + 32 * (warp >> 2)), v);
      tc::fence_before_sync();
      __syncwarp();
      if (lane == 0) tc::mbar_arrive(&tfree);
#pragma unroll
      for (int h = 0; h < 4; ++h) {  // 8 columns (16 words) per TMEM round trip
        uint32_t a[16];
        if (g > 0) {
          tc::tmem_ld16(tf64 + 16 * h, a);
        } else {
#pragma unroll
          for (int e = 0; e < 16; ++e) a[e] = 0u;
        }
#pragma unroll
        for (int e = 0; e < 8; ++e) {
          const double d =
              __hiloint2double((int)a[2 * e + 1], (int)a[2 * e]) + (double)v[8 * h + e];
          a[2 * e] = (uint32_t)__double2loint(d);
          a[2 * e + 1] = (uint32_t)__double2hiint(d);
        }
        tc::tmem_st16(tf64 + 16 * h, a);
      }
      tc::tmem_wait_st();  // the next read of the FP64 tile sees these
      return true;
    };

#pragma unroll
    for (int ch = 0; ch < NST - 1; ++ch) {
      if (ch < nch) load(ch, ch);
      tc::cp_commit();
    }
    int bad = 0;
    for (int ch = 0; ch < nch; ++ch) {
      tc::cp_wait<NST - 2>();
      // split buffer ch & 1 free once the MMAs of chunk ch - 2 are done
      const bool ok = ch < 2 || tc::mbar_wait_or(&done[ch & 1], ((ch - 2) >> 1) & 1, stop);
      if (tc::bar_or(WBAR, NW, bad || !ok)) {
        bad = 1;
        break;
      }
      convert(ch, ch % NST, ch & 1);
      tc::fence_async_shared();
      __syncwarp();
      if (lane == 0) tc::mbar_arrive(&full[ch & 1]);
      if (ch + NST - 1 < nch) load(ch + NST - 1, (ch + NST - 1) % NST);
      tc::cp_commit();
      if (ch >= 1 && (ch - 1) % NF == NF - 1 && !flush(ch - 1)) bad = 1;
    }
    if (!bad && nch > 0 && !flush(nch - 1)) bad = 1;
    if (tc::bar_or(WBAR, NW, bad)) *stop = 1;
    tc::cp_wait<0>();
  }

  tc::fence_before_sync();
  __syncthreads();
  const int failed = *stop;
  if (!failed && warp != MMA_WARP) {
    tc::fence_after_sync();
    if (DIAG && same) {  // the U units of row r sit in lanes l, l + 8, ... (same warp)
      double d = dacc;
#pragma unroll
      for (int m = 8; m < 8 * U; m <<= 1) d += __shfl_xor_sync(0xffffffffu, d, m);
      const int q = tid;  // A units: workers < 128 U
      if (q < ROWS * U && ((q >> 3) % U) == 0) diag_s[(q & 7) + 8 * ((q >> 3) / U)] = d;
      tc::bar_sync(WBAR, NW);
    }
    // ---- epilogue (workers): the FP64 tile plus the small terms' FP32
    // accumulator out of TMEM, 8 columns at a time
    const int rl = 32 * (warp & 3) + lane, cb = 32 * (warp >> 2);
    const uint32_t tsm = tbase + tlanes + (uint32_t)(32 * (warp >> 2));
    const double sc = MODE == 1 && r0 + rl < p.M
                          ? p.alpha * (p.w ? p.w[(r0 + rl) >> 1] : 1.0)
                          : 0.0;
#pragma unroll 1
    for (int pc = 0; pc < 4; ++pc) {
      uint32_t a[16], sm[8];
      double accs[8];
      tc::tmem_ld16(tf64 + 16 * pc, a);
      tc::tmem_ld8u(tsm + 8 * pc, sm);
#pragma unroll
      for (int e8 = 0; e8 < 8; ++e8) {
        const int e = 8 * pc + e8;
        const double acc = nch > 0 ? __hiloint2double((int)a[2 * e8 + 1], (int)a[2 * e8]) +
                                         (double)__uint_as_float(sm[e8])
                                   : 0.0;
        if (MODE == 0) {
          const int r = r0 + rl, c = c0 + cb + e;
          if (r < p.M && c < p.N)
            p.part[(size_t)blockIdx.z * p.M * p.N + (size_t)c * p.M + r] =
                (same && cb + e == rl) ? diag_s[rl] : acc;
        } else {
          accs[e8] = acc;
        }
      }
      if (MODE == 1) {
        // out = alpha w (acc [+ diag]) + beta out: every load of the piece is
        // issued before its first store, so their latencies overlap
        const int pt = r0 + rl;
        double ov[8], dg[8];
#pragma unroll
        for (int e8 = 0; e8 < 8; ++e8) {
          const int i = c0 + cb + 8 * pc + e8;
          const bool ok = pt < p.M && i < p.N;
          ov[e8] = (ok && p.beta != 0.0) ? p.out[(size_t)i * p.ldo + pt] : 0.0;
          dg[e8] = (MODE == 1 && ok && i < p.nin)
                       ? p.B[(size_t)i * p.ldb + i] * p.A[(size_t)i * p.lda + pt]
                       : 0.0;
        }
#pragma unroll
        for (int e8 = 0; e8 < 8; ++e8) {
          const int i = c0 + cb + 8 * pc + e8;
          if (pt < p.M && i < p.N) {
            const double v = sc * (accs[e8] + dg[e8]);
            p.out[(size_t)i * p.ldo + pt] = p.beta == 0.0 ? v : fma(p.beta, ov[e8], v);
          }
        }
      }
    }
  }
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) {
    tc::fence_after_sync();
    if (failed && issued_s > 0)  // nothing may still write TMEM when it is released
      tc::mbar_wait(&done[(issued_s - 1) & 1], ((issued_s - 1) >> 1) & 1);
    __syncwarp();
    tc::tmem_free(tbase, TMEM_COLS);
  }
  if (failed && tid == 0) atomicOr(p.err, 1);
}

template <int MODE, int NLD, int NST, int KC>
int launch(cudaStream_t s, dim3 grid, const Args& a) {
  using C = Cfg<MODE, NLD, NST, KC>;
  static_assert(C::BYTES + (int)sizeof(double) * ROWS + 128 <= 227 * 1024, "shared memory");
  static unsigned long long done = 0;  // per-device attribute, one bit per device
  int dev = 0;
  CPSTEP_CUDA_TRY(cudaGetDevice(&dev));
  const unsigned long long bit = 1ull << (dev & 63);
  if (!(__atomic_load_n(&done, __ATOMIC_ACQUIRE) & bit)) {
    CPSTEP_CUDA_TRY(cudaFuncSetAttribute(k_pc_tc<MODE, NLD, NST, KC>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, C::BYTES));
    __atomic_or_fetch(&done, bit, __ATOMIC_RELEASE);
  }
  k_pc_tc<MODE, NLD, NST, KC><<<grid, NTHR, C::BYTES, s>>>(a);
  CPSTEP_LAUNCH_CHECK();
  return CPSTEP_OK;
}

// overlap of one operand (S): 32-real chunks, 3 stages; two operands: 16-real
// chunks, 4 stages; one operand split in the CTA and one pre-split (MODE 1-3):
// 32-real chunks, 3 stages of each
constexpr int KC_ONE = 32, NST_ONE = 3, KC_TWO = 16, NST_TWO = 4, KC_PRE = 32, NST_PRE = 3;

inline bool al16(const void* q) { return ((uintptr_t)q & 15) == 0; }

// K steps per row tile of a pre-split operand (whole 32-real chunks) and its bytes
inline int pre_nsp(int K) { return cdiv(K, KC_PRE) * (KC_PRE / 16); }
inline size_t pre_bytes(int rows, int K) {
  return (size_t)cdiv(rows, ROWS) * (size_t)pre_nsp(K) * STEP_B;
}

int presplit(cpstep_ctx* c, const double* src, long long ldr, int rows, int K, const double* w,
             int zero_diag, uint8_t* dst) {
  if (!al16(src) || (ldr & 1) || rows < 1 || K < 1) return CPSTEP_ERR_ARG;
  PreArgs a{src, ldr, rows, K, pre_nsp(K), w, zero_diag, dst, nullptr};
  const long long threads = (long long)cdiv(rows, ROWS) * a.nsp * 8 * 32;
  k_presplit<<<(unsigned)((threads + 255) / 256), 256, 0, c->stream>>>(a);
  CPSTEP_LAUNCH_CHECK();
  return CPSTEP_OK;
}

// ---------------------------------------------------------------------------
// Back-multiply with a short inner dimension (nin <= 128, one fold group):
//   out[i][p] = alpha w(p) (sum_{j != i} M(j,i) in[j][p] + M(i,i) in[i][p]) + beta out[i][p]
// the same products, levels and summation order as k_pc_tc's MODE 1, sized
// for two CTAs per SM so that one CTA's epilogue (the output tile's stores)
// overlaps the other's operand loads: 16-real chunks, 8 worker warps that
// bring the FP64 rows in with cp.async (3 stages), split them into the BF16
// levels and write the tile; warp 8 issues the MMAs and streams the
// pre-split M^T in 3 stages.  TMEM holds the two FP32 accumulators only (256
// columns): with one fold group the hi*hi sum and the small products meet in
// FP64 in the epilogue, as the FP64 tile of k_pc_tc holds them after its
// first fold.
// The PsiV reset of the orthoT dynamics (CP_State_GSpacePlane.C:3707-3770,
// order 0) can ride on the epilogue of psi = psi_no.T: when *psiv_flag is
// set, v = (psi_new - psi_old) rdt and psi_no = psi_new.  The host passes it
// here only with one column tile (nout <= 128), where the CTA that writes a
// point of psi_no is the only one that reads it (many states: k_pp_tc's
// back-multiply epilogue).
constexpr int BM_NW = 256;                          // worker threads (warps 0-7)
constexpr int BM_MMA_WARP = BM_NW / 32;             // warp 8
constexpr int BM_NTHR = BM_NW + 32;
constexpr int BM_KC = 16;                           // reals (states) per chunk: one K step
constexpr int BM_OPB = STEP_B;                      // one operand of one chunk: 12 KB
constexpr int BM_NSTP = 3;                          // stages of the pre-split operand
constexpr int BM_NST = 3;                           // FP64 stages [KC][RSP]
constexpr int BM_RSP = ROWS + 2;
constexpr int BM_RAW = BM_KC * BM_RSP * 8;
constexpr int BM_BYTES = 1024 + 2 * BM_OPB + BM_NSTP * BM_OPB + BM_NST * BM_RAW;
constexpr uint32_t BM_TMEM_COLS = 2 * ROWS;
static_assert(2 * (BM_BYTES + 1024 + 128) <= 228 * 1024, "two CTAs per SM");
static_assert(BM_RAW % 16 == 0 && ROWS * (BM_KC / 8) == BM_NW, "one unit per worker");

struct BMArgs {
  const double* in;   // in[j][p], row j at in + j ldi
  const double* m;    // M column-major (column i at m + i ldm): the diagonal
  const uint8_t* pre; // B(i, j) = M(j, i) without the diagonal, k_presplit image
  const double* w;    // per complex point (a power of two), or none
  int ldi, ldm, ldo, pre_nsp;
  int np, nout, nin;  // points (reals), output rows, inner dimension (<= 128)
  double* out;
  double alpha, beta;
  const int* psiv_flag;  // PsiV reset: when set, v and psi_no from the new tile
  double* psiv_v;
  double* psiv_no;
  double rdt;
  int* err;
};

// Two CTAs per SM: 18 warps over the 4 SM sub-partitions put 5 on one, whose
// 16K registers then allow 102 per thread (the bound below).
__global__ void __launch_bounds__(BM_NTHR, 2) k_bm_tc(const BMArgs p) {
  extern __shared__ uint8_t dsm[];
  __shared__ uint64_t full[2], done[2], pfull[BM_NSTP];
  __shared__ uint32_t tslot;
  __shared__ int stop_s, issued_s;
  __shared__ double mdiag[ROWS];  // M(i, i) of the tile's columns
  volatile int* stop = &stop_s;
  const uint32_t s0 = tc::smem_u32(dsm);
  uint8_t* base = dsm + (((s0 + 1023u) & ~1023u) - s0);
  const uint32_t bf_s = tc::smem_u32(base);  // split A [2][level][4 KB]
  uint8_t* pre_base = base + 2 * BM_OPB;     // M^T stages [NSTP][level][4 KB]
  double* raw = reinterpret_cast<double*>(pre_base + BM_NSTP * BM_OPB);  // [NST][KC][RSP]
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int r0 = blockIdx.x * ROWS, c0 = blockIdx.y * ROWS;
  const int nch = (p.nin + BM_KC - 1) / BM_KC;  // 1 .. 8

  if (warp == 0) tc::tmem_alloc(&tslot, BM_TMEM_COLS);
  if (tid == 0) {
    for (int i = 0; i < 2; ++i) {
      tc::mbar_init(&full[i], BM_NW / 32);
      tc::mbar_init(&done[i], 1);
    }
    for (int i = 0; i < BM_NSTP; ++i) tc::mbar_init(&pfull[i], 1);
    stop_s = 0;
    issued_s = 0;
    tc::fence_mbar_init();
  }
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tbase = tslot;

  if (warp == BM_MMA_WARP) {
    if (lane == 0) {
      int bad = 0, issued = 0, req = 0;
      auto pre_load = [&](int c) {
        const int st = c % BM_NSTP;
        const uint8_t* src = p.pre + ((size_t)blockIdx.y * p.pre_nsp + (size_t)c) * STEP_B;
        tc::mbar_expect_tx(&pfull[st], BM_OPB);
        tc::bulk_g2s(pre_base + (size_t)st * BM_OPB, src, BM_OPB, &pfull[st]);
      };
      for (; req < nch && req < BM_NSTP; ++req) pre_load(req);
      for (int ch = 0; ch < nch; ++ch) {
        if (!tc::mbar_wait_or(&full[ch & 1], (ch >> 1) & 1, stop) ||
            !tc::mbar_wait_or(&pfull[ch % BM_NSTP], (ch / BM_NSTP) & 1, stop)) {
          bad = 1;
          break;
        }
        tc::fence_after_sync();
        const uint32_t a0 = bf_s + (uint32_t)((ch & 1) * BM_OPB);
        const uint32_t b0 = bf_s + (uint32_t)((2 + ch % BM_NSTP) * BM_OPB);
        // level pairs, smallest first; h h into its own accumulator
        constexpr int LA[6] = {2, 0, 1, 1, 0, 0};
        constexpr int LB[6] = {0, 2, 1, 0, 1, 0};
#pragma unroll
        for (int t = 0; t < 6; ++t) {
          const bool zero = ch == 0 && (t == 0 || t == 5);
          const uint64_t da = tc::smem_desc_kmajor(a0 + LA[t] * TILE_B, 128, 256);
          const uint64_t db = tc::smem_desc_kmajor(b0 + LB[t] * TILE_B, 128, 256);
          tc::mma_bf16(t == 5 ? tbase + ROWS : tbase, da, db, IDESC, zero ? 0u : 1u);
        }
        tc::commit(&done[ch & 1]);
        issued = ch + 1;
        if (ch >= 1 && req < nch) {  // chunk ch - 1's stage takes chunk req
          if (!tc::mbar_wait_or(&done[(ch - 1) & 1], ((ch - 1) >> 1) & 1, stop)) {
            bad = 1;
            break;
          }
          pre_load(req++);
        }
      }
      if (bad) {
        *stop = 1;
        for (int c = issued; c < req; ++c)  // requested copies land before the CTA exits
          tc::mbar_wait(&pfull[c % BM_NSTP], (c / BM_NSTP) & 1);
      }
      issued_s = issued;
    }
    __syncwarp();
  } else {
    // ---------------- workers
    // rows j = 16 ch .. of in (zero past nin), 128 points from r0 (zero past np)
    auto load = [&](int ch, int st) {
      double* ra = raw + (size_t)st * (BM_RAW / 8);
#pragma unroll
      for (int it = 0; it < BM_KC * (ROWS / 2) / BM_NW; ++it) {
        const int q = tid + BM_NW * it;
        const int jj = q / (ROWS / 2), pc = q % (ROWS / 2);
        const int j = ch * BM_KC + jj, pt = r0 + 2 * pc;
        const bool ok = j < p.nin && pt < p.np;  // np even: the pair is inside
        const double* g = ok ? p.in + (size_t)j * p.ldi + pt : p.in;
        tc::cp16(ra + jj * BM_RSP + 2 * pc, g, ok ? 16 : 0);
      }
    };
    if (tid < ROWS) {
      const int i = c0 + tid;
      mdiag[tid] = (i < p.nout && i < p.nin) ? p.m[(size_t)i * p.ldm + i] : 0.0;
    }
    // unit tid: row (point) r = (tid & 7) + 8 (tid >> 4), states 8 u .. (u = (tid >> 3) & 1)
    const int r = (tid & 7) + 8 * (tid >> 4), u = (tid >> 3) & 1;
#pragma unroll
    for (int ch = 0; ch < BM_NST - 1; ++ch) {
      if (ch < nch) load(ch, ch);
      tc::cp_commit();
    }
    int bad = 0;
    for (int ch = 0; ch < nch; ++ch) {
      tc::cp_wait<BM_NST - 2>();
      // split buffer ch & 1 is free once the MMAs of chunk ch - 2 are done
      const bool ok = ch < 2 || tc::mbar_wait_or(&done[ch & 1], ((ch - 2) >> 1) & 1, stop);
      if (tc::bar_or(WBAR, BM_NW, bad || !ok)) {
        bad = 1;
        break;
      }
      const double* ra = raw + (size_t)(ch % BM_NST) * (BM_RAW / 8);
      float f[8];
#pragma unroll
      for (int e = 0; e < 8; ++e) f[e] = (float)ra[(8 * u + e) * BM_RSP + r];
      split_store(base + (ch & 1) * BM_OPB + core_off(r, 8 * u), f);
      tc::fence_async_shared();
      __syncwarp();
      if (lane == 0) tc::mbar_arrive(&full[ch & 1]);
      if (ch + BM_NST - 1 < nch) load(ch + BM_NST - 1, (ch + BM_NST - 1) % BM_NST);
      tc::cp_commit();
    }
    if (!bad && !__all_sync(0xffffffffu,
                            tc::mbar_wait_or(&done[(nch - 1) & 1], ((nch - 1) >> 1) & 1, stop)))
      bad = 1;
    if (tc::bar_or(WBAR, BM_NW, bad)) *stop = 1;
    tc::cp_wait<0>();
  }

  tc::fence_before_sync();
  __syncthreads();
  const int failed = *stop;
  if (!failed && warp != BM_MMA_WARP) {
    tc::fence_after_sync();
    // warp w: TMEM lanes 32 (w % 4).. (rows = points), columns 64 (w / 4)..
    const uint32_t tlanes = (uint32_t)(32 * (warp & 3)) << 16;
    const int rl = 32 * (warp & 3) + lane, cb = 64 * (warp >> 2);
    const int pt = r0 + rl;
    const bool prow = pt < p.np;
    const double sc = prow ? p.alpha * (p.w ? p.w[pt >> 1] : 1.0) : 0.0;
    const bool pv = p.psiv_flag && *p.psiv_flag;
#pragma unroll 1
    for (int pc = 0; pc < 8; ++pc) {
      uint32_t sm[8], hh[8];
      tc::tmem_ld8u(tbase + tlanes + (uint32_t)(cb + 8 * pc), sm);
      tc::tmem_ld8u(tbase + tlanes + (uint32_t)(ROWS + cb + 8 * pc), hh);
      // every load of the piece is issued before its first store
      double ov[8], dg[8];
#pragma unroll
      for (int e8 = 0; e8 < 8; ++e8) {
        const int i = c0 + cb + 8 * pc + e8;
        const bool ok = prow && i < p.nout;
        ov[e8] = (ok && (p.beta != 0.0 || pv)) ? p.out[(size_t)i * p.ldo + pt] : 0.0;
        dg[e8] = (ok && i < p.nin) ? p.in[(size_t)i * p.ldi + pt] : 0.0;
      }
#pragma unroll
      for (int e8 = 0; e8 < 8; ++e8) {
        const int i = c0 + cb + 8 * pc + e8;
        if (prow && i < p.nout) {
          const double acc =
              (double)__uint_as_float(hh[e8]) + (double)__uint_as_float(sm[e8]);
          const double v = sc * fma(mdiag[cb + 8 * pc + e8], dg[e8], acc);
          const double o = p.beta == 0.0 ? v : fma(p.beta, ov[e8], v);
          p.out[(size_t)i * p.ldo + pt] = o;
          if (pv) {
            p.psiv_v[(size_t)i * p.ldo + pt] = (o - ov[e8]) * p.rdt;
            p.psiv_no[(size_t)i * p.ldi + pt] = o;
          }
        }
      }
    }
  }
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) {
    tc::fence_after_sync();
    if (failed && issued_s > 0)  // nothing may still write TMEM when it is released
      tc::mbar_wait(&done[(issued_s - 1) & 1], ((issued_s - 1) >> 1) & 1);
    __syncwarp();
    tc::tmem_free(tbase, BM_TMEM_COLS);
  }
  if (failed && tid == 0) atomicOr(p.err, 1);
}

// ---------------------------------------------------------------------------
// Products of two pre-split operands (FP16 levels of power-of-two scaled
// values, the k_presplit image): the EES sums with A = w psi dyp_c (rows
// c S + s) and B = the S rows of one atom type (rows v natm_t + a), and the
// PairCalc overlaps of many states (S, lambda), both operands split once in
// global memory.  No operand work is left in the CTA; the roles are
// warp-specialised:
//   warp 17 (lane 0)  streams each chunk's A and B levels with two bulk copies
//                     into one of PP_NST stages, as soon as the stage is free;
//   warp 16 (lane 0)  issues the 3 MMAs per K step (h m, m h, h h, all into one
//                     FP32 accumulator) as soon as a stage has landed, never
//                     waiting for MMAs to complete; the fold groups (nf chunks)
//                     alternate between two accumulator sets;
//   warps 0-15        add each finished group's accumulator into the FP64 tile
//                     (in TMEM for the FP16 images, in their registers, 32
//                     values per thread, for the BF16 ones) and write it.
//   part[ks][(c jp + j) S + s] = rinv[c] cinv[j] sum_{k in slab ks} A[c S + s][k] B[j][k]
// Handshakes (mbarriers, every wait bounded): full[st] (both copies of the
// stage landed), empty[st] (the MMAs that read it completed), gfull[b] (a
// group's MMAs into accumulator b completed), tfree[b] (accumulator b read
// back).
constexpr int PP_KC = 32;                     // reals per chunk (2 K steps)
constexpr int PP_KS = PP_KC / 16;
constexpr int PP_MMA_WARP = NW / 32, PP_LOAD_WARP = NW / 32 + 1;
constexpr int PP_NTHR = NW + 64;
// NL levels per element: 2 (FP16, scaled; 3 level products) or 3 (BF16; 6)
template <int NL>
struct PPCfg {
  static constexpr int STEP = NL * TILE_B;               // one K step, all levels
  static constexpr int OPB = PP_KS * STEP;               // one operand of one chunk
  static constexpr int STAGE = 2 * OPB;                  // A then B
  static constexpr int NST = NL == 2 ? 6 : 4;            // stages
  static constexpr int BYTES = 1024 + NST * STAGE;
  static_assert(NST * STAGE >= (128 * 129 + 128) * 8, "back-multiply tile in the stages");
  static constexpr int NPROD = NL == 2 ? 3 : 6;
  // TMEM, two fold groups in flight: FP16 one accumulator per group (columns
  // 0-255) and the FP64 tile in columns 256-511; BF16 two per group, the h h
  // product apart from the five small ones (all 512 columns), and the FP64
  // tile in the fold warps' registers
  static constexpr int NSLOT = NL == 2 ? 1 : 2;
  static constexpr int NGRP = 2;
};

struct PPArgs {
  const uint8_t* a;  // [row tile][K step][level][4 KB], nsp K steps per row tile
  const uint8_t* b;
  int nsp;
  int M, N, K;       // rows of A (nch S), rows of B (jp), reals
  int kslab;         // reals per split (whole fold groups: 512 reals FP16, 128 BF16)
  int S, jp;         // states (rows of one channel block of A), B rows per channel block
  float rinv[4];     // 1 / scale of A's channel blocks
  const float* cinv; // 1 / scale of B row j at cinv[j cstride] (device), or none (1)
  int cstride;       // 1, or 0 for one scale of every row
  double* part;      // [nsplit][nch jp][S]
  int* err;
  // back-multiply epilogue (BM): A = in^T (rows = points' reals), B = M^T
  // without its diagonal, K = nin; out[i][p] = alpha w(p) (D[p][i] + M(i,i)
  // in[i][p]) + beta out[i][p]
  const double* in;
  const double* m;
  const double* w;
  double* out;
  int ldi, ldm, ldo;
  double alpha, beta;
  // the PsiV reset of psi = psi_no.T (as k_bm_tc): when *psiv_flag, v = (new -
  // old) rdt and psi_no = new.  in is read in the kernel only at the points and
  // states a CTA writes (the diagonal term), so any number of column tiles may
  // write psi_no = in.
  const int* psiv_flag;
  double* psiv_v;
  double rdt;
};

template <int NL, bool BM>
__global__ void __launch_bounds__(PP_NTHR, 1) k_pp_tc(const PPArgs p) {
  using C = PPCfg<NL>;
  constexpr int PP_NST = C::NST, PP_OPB = C::OPB, PP_STAGE = C::STAGE, STEP = C::STEP;
  extern __shared__ uint8_t dsm[];
  constexpr int NGRP = C::NGRP, NSLOT = C::NSLOT;
  __shared__ uint64_t full[PP_NST], empty[PP_NST], gfull[NGRP], tfree[NGRP];
  __shared__ uint32_t tslot;
  __shared__ int stop_s, issued_s, req_s;
  volatile int* stop = &stop_s;
  const uint32_t s0 = tc::smem_u32(dsm);
  uint8_t* base = dsm + (((s0 + 1023u) & ~1023u) - s0);
  const uint32_t base_s = tc::smem_u32(base);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  // row and column tile; the back-multiply runs the column tiles of a point
  // tile side by side (grid x), so that they read its A levels from L2
  const int rt = BM ? blockIdx.y : blockIdx.x, ct = BM ? blockIdx.x : blockIdx.y;
  const int r0 = rt * ROWS, c0 = ct * ROWS;
  const int kbeg = blockIdx.z * p.kslab, kend = min(p.K, kbeg + p.kslab);
  const int nch = kend > kbeg ? (kend - kbeg + PP_KC - 1) / PP_KC : 0;
  constexpr int nf = NL == 2 ? 512 / PP_KC : 128 / PP_KC;  // chunks per fold group
  const int ngroups = (nch + nf - 1) / nf;

  if (warp == 0) tc::tmem_alloc(&tslot, TMEM_COLS);
  if (tid == 0) {
    for (int i = 0; i < PP_NST; ++i) {
      tc::mbar_init(&full[i], 1);
      tc::mbar_init(&empty[i], 1);
    }
    for (int i = 0; i < NGRP; ++i) {
      tc::mbar_init(&gfull[i], 1);
      tc::mbar_init(&tfree[i], NW / 32);
    }
    stop_s = 0;
    issued_s = 0;
    req_s = 0;
    tc::fence_mbar_init();
  }
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tbase = tslot;
  const uint32_t tlanes = (uint32_t)(32 * (warp & 3)) << 16;
  // FP16 images: the FP64 tile in TMEM columns 256-511; BF16: in the workers'
  // registers (row 32 (warp % 4) + lane, columns 32 (warp / 4)..)
  const uint32_t tf64 = tbase + tlanes + TMEM_F64 + (uint32_t)(64 * ((warp >> 2) & 3));
  double acc64[NL == 2 ? 1 : 32];

  if (warp == PP_LOAD_WARP) {
    if (lane == 0) {
      int req = 0;
      for (; req < nch; ++req) {
        const int st = req % PP_NST;
        if (req >= PP_NST &&  // the MMAs of chunk req - PP_NST read this stage
            !tc::mbar_wait_fast(&empty[st], ((req - PP_NST) / PP_NST) & 1, stop)) {
          *stop = 1;
          break;
        }
        const size_t kstep = (size_t)((kbeg + req * PP_KC) >> 4);
        const uint8_t* ga = p.a + ((size_t)rt * p.nsp + kstep) * STEP;
        const uint8_t* gb = p.b + ((size_t)ct * p.nsp + kstep) * STEP;
        uint8_t* sa = base + (size_t)st * PP_STAGE;
        tc::mbar_expect_tx(&full[st], PP_STAGE);
        tc::bulk_g2s(sa, ga, PP_OPB, &full[st]);
        tc::bulk_g2s(sa + PP_OPB, gb, PP_OPB, &full[st]);
      }
      req_s = req;
    }
    __syncwarp();
  } else if (warp == PP_MMA_WARP) {
    if (lane == 0) {
      int issued = 0;
      for (int c = 0; c < nch; ++c) {
        const int st = c % PP_NST, g = c / nf, acc = g % NGRP;
        const bool first = c % nf == 0;
        if (first && g >= NGRP) {  // accumulator set acc was folded (group g - NGRP)
          if (!tc::mbar_wait_fast(&tfree[acc], ((g - NGRP) / NGRP) & 1, stop)) break;
          tc::fence_after_sync();
        }
        if (!tc::mbar_wait_fast(&full[st], (c / PP_NST) & 1, stop)) break;
        tc::fence_after_sync();
        const uint32_t a0 = base_s + (uint32_t)(st * PP_STAGE), b0 = a0 + PP_OPB;
        // level pairs, smallest first: FP16 (m, h), (h, m), (h, h); BF16 as k_pc_tc's six
        constexpr int LA2[3] = {1, 0, 0}, LB2[3] = {0, 1, 0};
        constexpr int LA3[6] = {2, 0, 1, 1, 0, 0}, LB3[6] = {0, 2, 1, 0, 1, 0};
#pragma unroll
        for (int s = 0; s < PP_KS; ++s) {
#pragma unroll
          for (int t = 0; t < C::NPROD; ++t) {
            const int la = NL == 2 ? LA2[t % 3] : LA3[t], lb = NL == 2 ? LB2[t % 3] : LB3[t];
            const uint64_t da = tc::smem_desc_kmajor(a0 + s * STEP + la * TILE_B, 128, 256);
            const uint64_t db = tc::smem_desc_kmajor(b0 + s * STEP + lb * TILE_B, 128, 256);
            const bool hh = NL == 3 && t == 5;  // BF16: h h into the set's second slot
            const bool zero = first && s == 0 && (t == 0 || hh);
            tc::mma_bf16(tbase + (uint32_t)((NSLOT * acc + (hh ? 1 : 0)) * ROWS), da, db,
                         NL == 2 ? IDESC_H : IDESC, zero ? 0u : 1u);
          }
        }
        tc::commit(&empty[st]);
        if (c % nf == nf - 1 || c == nch - 1) tc::commit(&gfull[acc]);
        issued = c + 1;
      }
      if (issued < nch) *stop = 1;
      issued_s = issued;
    }
    __syncwarp();
  } else {
#pragma unroll
    for (int e = 0; e < (NL == 2 ? 1 : 32); ++e) acc64[e] = 0.0;
    int bad = 0;
    for (int g = 0; g < ngroups && !bad; ++g) {
      const int acc = g % NGRP;
      if (!__all_sync(0xffffffffu, tc::mbar_wait_fast(&gfull[acc], (g / NGRP) & 1, stop))) {
        bad = 1;
        break;
      }
      tc::fence_after_sync();
      const uint32_t ta = tbase + tlanes + (uint32_t)(NSLOT * acc * ROWS + 32 * (warp >> 2));
      if constexpr (NL == 2) {
        // the accumulator read back and released, then added into the FP64
        // tile in TMEM columns 256-511, 8 columns (16 words) per round trip
        float v[32];
        tc::tmem_ld32(ta, v);
        tc::fence_before_sync();
        __syncwarp();
        if (lane == 0) tc::mbar_arrive(&tfree[acc]);
#pragma unroll
        for (int h = 0; h < 4; ++h) {
          uint32_t a[16];
          if (g > 0) {
            tc::tmem_ld16(tf64 + 16 * h, a);
          } else {
#pragma unroll
            for (int e = 0; e < 16; ++e) a[e] = 0u;
          }
#pragma unroll
          for (int e = 0; e < 8; ++e) {
            const double d =
                __hiloint2double((int)a[2 * e + 1], (int)a[2 * e]) + (double)v[8 * h + e];
            a[2 * e] = (uint32_t)__double2loint(d);
            a[2 * e + 1] = (uint32_t)__double2hiint(d);
          }
          tc::tmem_st16(tf64 + 16 * h, a);
        }
        tc::tmem_wait_st();  // the next read of the FP64 tile sees these
        continue;
      } else {
#pragma unroll
        for (int h = 0; h < 4; ++h) {  // 8 columns of both slots at a time
          uint32_t v0[8], v1[8];
          tc::tmem_ld8u(ta + 8 * h, v0);
          tc::tmem_ld8u(ta + ROWS + 8 * h, v1);
#pragma unroll
          for (int e = 0; e < 8; ++e)
            acc64[(8 * h + e) % (NL == 2 ? 1 : 32)] +=
                (double)__uint_as_float(v1[e]) + (double)__uint_as_float(v0[e]);
        }
      }
      tc::fence_before_sync();
      __syncwarp();
      if (lane == 0) tc::mbar_arrive(&tfree[acc]);
    }
    if (tc::bar_or(WBAR, NW, bad)) *stop = 1;
  }

  tc::fence_before_sync();
  __syncthreads();
  const int failed = *stop;
  if (BM && !failed && warp < PP_MMA_WARP && nch > 0) {
    // rows = points, columns = output states: the FP64 tile through the (now
    // idle) stage buffers, then written point-contiguous
    double* tile = reinterpret_cast<double*>(base);  // [128][129]
    double* mdg = tile + ROWS * (ROWS + 1);          // M(i, i) of the tile's columns
    const int rl = 32 * (warp & 3) + lane, cb = 32 * (warp >> 2);
#pragma unroll
    for (int e = 0; e < 32; ++e) tile[rl * (ROWS + 1) + cb + e] = acc64[e % (NL == 2 ? 1 : 32)];
    if (tid < ROWS) {
      const int i = c0 + tid;
      mdg[tid] = (i < p.N && i < p.K) ? p.m[(size_t)i * p.ldm + i] : 0.0;
    }
    tc::bar_sync(WBAR, NW);
    const bool pv = p.psiv_flag && *p.psiv_flag;
    const bool rd = p.beta != 0.0 || pv;
    const int pl = tid % ROWS, il0 = tid / ROWS;  // this thread: point pl, columns il0 + 4 k
    const int pt = r0 + pl;
    const double sc = pt < p.M ? p.alpha * (p.w ? p.w[pt >> 1] : 1.0) : 0.0;
    // 32 elements per thread in two batches of 16: every load of a batch is
    // issued before its first store (a store to out or, with the PsiV reset,
    // to in would otherwise hold each next load back)
#pragma unroll
    for (int bt = 0; bt < 2; ++bt) {
      double dg[16], ov[16];
#pragma unroll
      for (int k = 0; k < 16; ++k) {
        const int il = il0 + 4 * (16 * bt + k), i = c0 + il;
        const bool ok = i < p.N && pt < p.M;
        dg[k] = (ok && i < p.K) ? p.in[(size_t)i * p.ldi + pt] : 0.0;
        ov[k] = (ok && rd) ? p.out[(size_t)i * p.ldo + pt] : 0.0;
      }
#pragma unroll
      for (int k = 0; k < 16; ++k) {
        const int il = il0 + 4 * (16 * bt + k), i = c0 + il;
        if (i < p.N && pt < p.M) {
          const double v = sc * fma(mdg[il], dg[k], tile[pl * (ROWS + 1) + il]);
          const double o = p.beta == 0.0 ? v : fma(p.beta, ov[k], v);
          p.out[(size_t)i * p.ldo + pt] = o;
          if (pv) {
            p.psiv_v[(size_t)i * p.ldo + pt] = (o - ov[k]) * p.rdt;
            const_cast<double*>(p.in)[(size_t)i * p.ldi + pt] = o;
          }
        }
      }
    }
  }
  if (!BM && !failed && warp < PP_MMA_WARP && nch > 0) {
    const int rl = 32 * (warp & 3) + lane, cb = 32 * (warp >> 2);
    const int r = r0 + rl;
    const int ch = r < p.M ? r / p.S : 0, s = r - ch * p.S;
    const double ri =
        (double)(ch == 0 ? p.rinv[0] : ch == 1 ? p.rinv[1] : ch == 2 ? p.rinv[2] : p.rinv[3]);
    double* out = p.part + (size_t)blockIdx.z * p.M * p.N + (size_t)ch * p.jp * p.S + s;
    if constexpr (NL == 2) {
      tc::fence_after_sync();
#pragma unroll 1
      for (int pc = 0; pc < 4; ++pc) {
        uint32_t a[16];
        tc::tmem_ld16(tf64 + 16 * pc, a);
#pragma unroll
        for (int e8 = 0; e8 < 8; ++e8) {
          const int j = c0 + cb + 8 * pc + e8;
          if (r < p.M && j < p.N)
            out[(size_t)j * p.S] = __hiloint2double((int)a[2 * e8 + 1], (int)a[2 * e8]) * ri *
                                   (p.cinv ? (double)p.cinv[j * p.cstride] : 1.0);
        }
      }
    } else {
#pragma unroll
      for (int e = 0; e < 32; ++e) {
        const int j = c0 + cb + e;
        if (r < p.M && j < p.N)
          out[(size_t)j * p.S] =
              acc64[e % (NL == 2 ? 1 : 32)] * ri * (p.cinv ? (double)p.cinv[j * p.cstride] : 1.0);
      }
    }
  }
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) {
    tc::fence_after_sync();
    if (failed) {
      // requested copies land and issued MMAs complete before the CTA exits
      for (int c = issued_s; c < req_s; ++c) tc::mbar_wait(&full[c % PP_NST], (c / PP_NST) & 1);
      if (issued_s > 0)
        tc::mbar_wait(&empty[(issued_s - 1) % PP_NST], ((issued_s - 1) / PP_NST) & 1);
    }
    __syncwarp();
    tc::tmem_free(tbase, TMEM_COLS);
  }
  if (failed && tid == 0) atomicOr(p.err, 1);
}

// The diagonal of S = overlap(psi, psi) for the many-state overlap: the
// FP64 row sums of w x^2, one block per row (fixed order).
__global__ void __launch_bounds__(256) k_rowdot(const double* __restrict__ src, long long ldr,
                                                int K, const double* __restrict__ w,
                                                double* __restrict__ diag) {
  __shared__ double red[32];
  const double* x = src + (size_t)blockIdx.x * ldr;
  double d = 0.0;
  for (int k2 = threadIdx.x; 2 * k2 < K; k2 += blockDim.x) {  // point k2: reals 2 k2, 2 k2 + 1
    const double2 v = *reinterpret_cast<const double2*>(x + 2 * k2);
    const double ww = w ? w[k2] : 1.0;
    d = fma(ww * v.x, v.x, fma(ww * v.y, v.y, d));
  }
  d = block_sum(d, red);
  if (threadIdx.x == 0) diag[blockIdx.x] = d;
}

// A of a many-state back-multiply: in^T (rows = the points' reals p, K =
// states j) as three BF16 levels in the k_presplit image.  Mapping as
// k_presplit; a lane reads its 8 states of one point, the warp's lanes
// consecutive points (64-byte runs).
__global__ void __launch_bounds__(256) k_presplit_t(const double* __restrict__ in, long long ldi,
                                                    int np, int nin, int nsp,
                                                    uint8_t* __restrict__ dst) {
  const long long wid = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  const long long nwarps = (long long)cdiv(np, ROWS) * nsp * 8;
  if (wid >= nwarps) return;
  const int gp = (int)(wid % 8);
  const long long rest = wid / 8;
  const int st = (int)(rest % nsp);
  const long long rt = rest / nsp;
  const int rl = (lane & 7) + 8 * (lane >> 4) + 16 * gp;
  const int kh = (lane >> 3) & 1;
  const long long pt = rt * ROWS + rl;
  const int j0 = 16 * st + 8 * kh;
  double x[8];
#pragma unroll
  for (int e = 0; e < 8; ++e) {
    const int j = j0 + e;
    x[e] = (pt < np && j < nin) ? in[(size_t)j * ldi + pt] : 0.0;
  }
  const float one[4] = {1.f, 1.f, 1.f, 1.f};
  float f[8];
  to_f32(x, one, f);
  split_store(dst + ((size_t)rt * nsp + st) * STEP_B + core_off(rl, 8 * kh), f);
}

// A of the EES sums of up to two atom types: rows c S + s (c < nch[t], s < S)
// = w psi_s dyp_{t,c} (complex, real view), scaled by sig[t][c] (a power of
// two), two FP16 levels in the k_presplit image at dst[t]; rows past nch S
// and reals past K are zero.  One warp = 16 states x 16 reals of one K step
// for every channel of every type: psi is read once.
struct PreA {
  const double* psi;  // [S][K] reals
  const double* w;    // per point (1 or 2)
  int ntyp;           // 1 or 2
  const float2* dyp[2];  // type t, channel c at dyp[t] + c ld_d
  int ld_d;
  int S, K, nsp;
  int nch[2];
  float sig[2][4];
  uint8_t* dst[2];
  int* err;
};
__global__ void __launch_bounds__(256) k_presplit_ees_a(const PreA a) {
  const long long wid = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  const int stiles = cdiv(a.S, ROWS);
  const long long nwarps = (long long)stiles * a.nsp * 8;
  if (wid >= nwarps) return;
  const int gp = (int)(wid % 8);
  const long long rest = wid / 8;
  const int st = (int)(rest % a.nsp);
  const int rt = (int)(rest / a.nsp);
  const int sl = (lane & 7) + 8 * (lane >> 4) + 16 * gp;
  const int kh = (lane >> 3) & 1;
  const int s = rt * ROWS + sl;
  const int k0 = 16 * st + 8 * kh;  // first real; 4 points from k0 / 2
  float xr[4], xi[4];
#pragma unroll
  for (int e = 0; e < 4; ++e) {
    const int pt = (k0 >> 1) + e;
    const bool ok = s < a.S && 2 * pt < a.K;
    const double2 x = ok ? *reinterpret_cast<const double2*>(a.psi + (size_t)s * a.K + 2 * pt)
                         : make_double2(0.0, 0.0);
    const float ws = ok ? (float)a.w[pt] : 0.f;
    xr[e] = (float)x.x * ws;
    xi[e] = (float)x.y * ws;
  }
  bool big = false;
#pragma unroll
  for (int t = 0; t < 2; ++t) {
    if (t >= a.ntyp) break;
    const float2* dyp = t == 0 ? a.dyp[0] : a.dyp[1];
    const int nch = t == 0 ? a.nch[0] : a.nch[1];
    uint8_t* dst = t == 0 ? a.dst[0] : a.dst[1];
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      if (c >= nch) break;
      float f[8];
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const int pt = (k0 >> 1) + e;
        const float2 d = 2 * pt < a.K ? dyp[(size_t)c * a.ld_d + pt] : make_float2(0.f, 0.f);
        f[2 * e] = fmaf(xr[e], d.x, -xi[e] * d.y);
        f[2 * e + 1] = fmaf(xr[e], d.y, xi[e] * d.x);
      }
      const float sc = t == 0 ? a.sig[0][c] : a.sig[1][c];
#pragma unroll
      for (int e = 0; e < 8; ++e) big |= !(fabsf(f[e] * sc) < 32768.f);
      if (s < a.S) {  // row c S + s of A; rows past nch S are never read into the output
        const int r = c * a.S + s;
        split_store_h(dst + ((size_t)(r / ROWS) * a.nsp + st) * STEP_H + core_off(r % ROWS, 8 * kh),
                      f, sc);
      }
    }
  }
  if (big) atomicOr(a.err, 4);
}

// ---------------------------------------------------------------------------
// psi force of up to two atom types from pre-split operands:
//   F_s(p) += alpha w(p) sum_t sum_c conj(dyp_tc(p)) Q_tcs(p),
//   Q_tcs(p) = sum_{a in t} Z_t(c natm_t + a, s) S_a(p)
// as D_t = A_t B_t^T with A_t = Z_t (rows 4 s + c, K = the type's atoms) and
// B_t = the real views of the type's S (Mn) rows transposed (rows = reals of
// the points, K = atoms), both FP16 levels (k_presplit_z, k_presplit_st).  One
// output tile = 32 states x 4 channel rows x 128 reals (64 points); the CTAs
// of one row tile walk the point tiles (persistent), the K chunks of a tile
// (the first type's, then the second's, each into its own accumulator)
// streamed like k_pp_tc's (warp 17 copies, warp 16 issues; two tiles in
// flight), and warps 0-15 finish each tile: the channel rows of a state are
// combined by lane shuffles, the types added, and F read and written once.
constexpr int PF_KC = 64;                 // atoms per chunk (4 K steps)
constexpr int PF_KS = PF_KC / 16;
constexpr int PF_OPB = PF_KS * STEP_H;    // 32 KB
constexpr int PF_STAGE = 2 * PF_OPB;      // 64 KB
constexpr int PF_NST = 3;
constexpr int PF_BYTES = 1024 + PF_NST * PF_STAGE;
constexpr uint32_t PF_TMEM_COLS = 4 * ROWS;  // [tile parity][type] accumulators

struct PFArgs {
  int ntyp;              // 1 or 2
  const uint8_t* a[2];   // Z levels of type t [row tile][K step][level][4 KB], nks[t] K steps
  const uint8_t* b[2];   // S^T levels of type t, the same image over the point reals
  int nks[2];            // K steps of type t: cdiv(natm_t, 16)
  int nch[2];
  const float* zmax[2];  // the FP16 scales of Z_t (pow2_scale(*zmax[t])) and of S^T_t
  const float* smax[2];  // (pow2_scale(*smax[t])), as k_presplit_z / k_presplit_st
  const float2* dyp[2];  // type t, channel c at dyp[t] + c ld_d (FP32)
  int ntile;             // row tiles of B (point tiles)
  int S, npts, ld_d;
  const double* w;       // per point
  double alpha;
  double* f;             // [S][2 npts] (+=)
  int* err;
};

__global__ void __launch_bounds__(PP_NTHR, 1) k_pf_tc(const PFArgs p) {
  extern __shared__ uint8_t dsm[];
  __shared__ uint64_t full[PF_NST], empty[PF_NST], gfull[2], tfree[2];
  __shared__ uint32_t tslot;
  __shared__ int stop_s, issued_s, req_s;
  volatile int* stop = &stop_s;
  const uint32_t s0 = tc::smem_u32(dsm);
  uint8_t* base = dsm + (((s0 + 1023u) & ~1023u) - s0);
  const uint32_t base_s = tc::smem_u32(base);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int m = blockIdx.y;
  const int ntyp = p.ntyp;
  const int nkc0 = (p.nks[0] + PF_KS - 1) / PF_KS;                   // K chunks per tile, type 0
  const int nkc1 = ntyp > 1 ? (p.nks[1] + PF_KS - 1) / PF_KS : 0;    // type 1
  // this CTA's point tiles: blockIdx.x, + gridDim.x, ...
  const int ntl = p.ntile > (int)blockIdx.x ? (p.ntile - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;
  const int nitem = ntl * (nkc0 + nkc1);

  if (warp == 0) tc::tmem_alloc(&tslot, PF_TMEM_COLS);
  if (tid == 0) {
    for (int i = 0; i < PF_NST; ++i) {
      tc::mbar_init(&full[i], 1);
      tc::mbar_init(&empty[i], 1);
    }
    for (int i = 0; i < 2; ++i) {
      tc::mbar_init(&gfull[i], 1);
      tc::mbar_init(&tfree[i], NW / 32);
    }
    stop_s = 0;
    issued_s = 0;
    req_s = 0;
    tc::fence_mbar_init();
  }
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tbase = tslot;
  const uint32_t tlanes = (uint32_t)(32 * (warp & 3)) << 16;

  if (warp == PP_LOAD_WARP) {
    if (lane == 0) {
      int req = 0;
      bool bad = false;
      for (int tl = 0; tl < ntl && !bad; ++tl) {
        const int n = blockIdx.x + tl * gridDim.x;
        for (int t = 0; t < ntyp && !bad; ++t) {
          const int nkc = t == 0 ? nkc0 : nkc1, nks = t == 0 ? p.nks[0] : p.nks[1];
          const uint8_t* ga = t == 0 ? p.a[0] : p.a[1];
          const uint8_t* gb = t == 0 ? p.b[0] : p.b[1];
          for (int kc = 0; kc < nkc; ++kc, ++req) {
            const int st = req % PF_NST;
            if (req >= PF_NST &&
                !tc::mbar_wait_fast(&empty[st], ((req - PF_NST) / PF_NST) & 1, stop)) {
              *stop = 1;
              bad = true;
              break;
            }
            const int ks0 = kc * PF_KS, ksz = min(PF_KS, nks - ks0);
            const uint32_t bytes = (uint32_t)ksz * STEP_H;
            uint8_t* sa = base + (size_t)st * PF_STAGE;
            tc::mbar_expect_tx(&full[st], 2 * bytes);
            tc::bulk_g2s(sa, ga + ((size_t)m * nks + ks0) * STEP_H, bytes, &full[st]);
            tc::bulk_g2s(sa + PF_OPB, gb + ((size_t)n * nks + ks0) * STEP_H, bytes, &full[st]);
          }
        }
      }
      req_s = req;
    }
    __syncwarp();
  } else if (warp == PP_MMA_WARP) {
    if (lane == 0) {
      int it = 0;
      bool bad = false;
      for (int tl = 0; tl < ntl && !bad; ++tl) {
        const int acc = tl & 1;
        for (int t = 0; t < ntyp && !bad; ++t) {
          const int nkc = t == 0 ? nkc0 : nkc1, nks = t == 0 ? p.nks[0] : p.nks[1];
          for (int kc = 0; kc < nkc; ++kc, ++it) {
            const int st = it % PF_NST;
            if (t == 0 && kc == 0 && tl >= 2) {  // accumulator pair acc read back (tile tl - 2)
              if (!tc::mbar_wait_fast(&tfree[acc], ((tl - 2) >> 1) & 1, stop)) {
                bad = true;
                break;
              }
              tc::fence_after_sync();
            }
            if (!tc::mbar_wait_fast(&full[st], (it / PF_NST) & 1, stop)) {
              bad = true;
              break;
            }
            tc::fence_after_sync();
            const int ksz = min(PF_KS, nks - kc * PF_KS);
            const uint32_t a0 = base_s + (uint32_t)(st * PF_STAGE), b0 = a0 + PF_OPB;
            const uint32_t d = tbase + (uint32_t)((2 * acc + t) * ROWS);
            for (int s = 0; s < ksz; ++s) {
#pragma unroll
              for (int q = 0; q < 3; ++q) {
                const int la = q == 0 ? 1 : 0, lb = q == 1 ? 1 : 0;  // (m, h), (h, m), (h, h)
                const uint64_t da = tc::smem_desc_kmajor(a0 + s * STEP_H + la * TILE_B, 128, 256);
                const uint64_t db = tc::smem_desc_kmajor(b0 + s * STEP_H + lb * TILE_B, 128, 256);
                const bool zero = kc == 0 && s == 0 && q == 0;
                tc::mma_bf16(d, da, db, IDESC_H, zero ? 0u : 1u);
              }
            }
            tc::commit(&empty[st]);
            if (t == ntyp - 1 && kc == nkc - 1) tc::commit(&gfull[acc]);
          }
        }
      }
      if (it < nitem) *stop = 1;
      issued_s = it;
    }
    __syncwarp();
  } else {
    // rows 4 s + c of this warp's lanes; columns (reals) 32 (warp / 4).. of the tile
    const int rl = 32 * (warp & 3) + lane;
    const int rg = m * ROWS + rl, s = rg >> 2, c = rg & 3;
    // 1 / (Z scale x S^T scale) of each type: powers of two, folded into dyp exactly
    float rinv[2];
#pragma unroll
    for (int t = 0; t < 2; ++t)
      rinv[t] = t < ntyp ? 1.f / (tc::pow2_scale(*p.zmax[t]) * tc::pow2_scale(*p.smax[t])) : 0.f;
    int bad = 0;
    for (int tl = 0; tl < ntl && !bad; ++tl) {
      const int acc = tl & 1;
      if (!__all_sync(0xffffffffu, tc::mbar_wait_fast(&gfull[acc], (tl >> 1) & 1, stop))) {
        bad = 1;
        break;
      }
      tc::fence_after_sync();
      const int n = blockIdx.x + tl * gridDim.x;
      const int pt0 = (n * ROWS + 32 * (warp >> 2)) >> 1;  // 16 points
      // conj(dyp_tc) Q_tcs summed over the state's 4 channel lanes (shuffles)
      // and the types; then lane c of the state adds points pt0 + c, + 4, + 8,
      // + 12 into F
      const bool wr = s < p.S;
      double2* fr = reinterpret_cast<double2*>(p.f + (size_t)(wr ? s : 0) * 2 * p.npts);
      float ox4[4] = {0.f, 0.f, 0.f, 0.f}, oy4[4] = {0.f, 0.f, 0.f, 0.f};
      double2 fo[4];
      for (int t = 0; t < ntyp; ++t) {
        if (t == ntyp - 1) {  // F's loads in flight during the last type's products
#pragma unroll
          for (int e4 = 0; e4 < 4; ++e4) {
            const int pt = pt0 + 4 * e4 + c;
            fo[e4] = (wr && pt < p.npts) ? fr[pt] : make_double2(0.0, 0.0);
          }
        }
        const bool live = s < p.S && c < (t == 0 ? p.nch[0] : p.nch[1]);
        const float2* dyp = t == 0 ? p.dyp[0] : p.dyp[1];
        const float ri = t == 0 ? rinv[0] : rinv[1];
#pragma unroll
        for (int hf = 0; hf < 2; ++hf) {  // 8 points (16 columns) at a time
          float2 d[8];
#pragma unroll
          for (int e = 0; e < 8; ++e) {
            const int pt = pt0 + 8 * hf + e;
            const float2 q = (live && pt < p.npts) ? dyp[(size_t)c * p.ld_d + pt]
                                                   : make_float2(0.f, 0.f);
            d[e] = make_float2(q.x * ri, q.y * ri);
          }
          uint32_t v[16];
          tc::tmem_ld16(tbase + tlanes + (uint32_t)((2 * acc + t) * ROWS + 32 * (warp >> 2) + 16 * hf),
                        v);
#pragma unroll
          for (int e = 0; e < 8; ++e) {
            const float qx = __uint_as_float(v[2 * e]), qy = __uint_as_float(v[2 * e + 1]);
            float ox = fmaf(d[e].x, qx, d[e].y * qy), oy = fmaf(d[e].x, qy, -d[e].y * qx);
            ox += __shfl_xor_sync(0xffffffffu, ox, 1);
            oy += __shfl_xor_sync(0xffffffffu, oy, 1);
            ox += __shfl_xor_sync(0xffffffffu, ox, 2);
            oy += __shfl_xor_sync(0xffffffffu, oy, 2);
            if ((e & 3) == c) {  // compile-time e, runtime c: keep this lane's four
              ox4[2 * hf + (e >> 2)] += ox;
              oy4[2 * hf + (e >> 2)] += oy;
            }
          }
        }
      }
      tc::fence_before_sync();
      __syncwarp();
      if (lane == 0) tc::mbar_arrive(&tfree[acc]);
#pragma unroll
      for (int e4 = 0; e4 < 4; ++e4) {
        const int pt = pt0 + 4 * e4 + c;
        if (wr && pt < p.npts) {
          const double sc = p.alpha * p.w[pt];
          fr[pt] = make_double2(fma(sc, (double)ox4[e4], fo[e4].x), fma(sc, (double)oy4[e4], fo[e4].y));
        }
      }
    }
    if (tc::bar_or(WBAR, NW, bad)) *stop = 1;
  }
  tc::fence_before_sync();
  __syncthreads();
  const int failed = *stop;
  if (warp == 0) {
    tc::fence_after_sync();
    if (failed) {
      for (int c = issued_s; c < req_s; ++c) tc::mbar_wait(&full[c % PF_NST], (c / PF_NST) & 1);
      if (issued_s > 0)
        tc::mbar_wait(&empty[(issued_s - 1) % PF_NST], ((issued_s - 1) / PF_NST) & 1);
    }
    __syncwarp();
    tc::tmem_free(tbase, PF_TMEM_COLS);
  }
  if (failed && tid == 0) atomicOr(p.err, 1);
}

// Z levels for k_pf_tc: rows 4 s + c (zero for c >= nch or s >= S), K = the
// type's atoms a (zero past natm_t): Z(c natm_t + a, s) = zt[s ldz + c natm_t
// + a], scaled by pow2_scale(*zmax).  One thread = 8 atoms of one row.
__global__ void k_presplit_z(const double* __restrict__ zt, int ldz, int S, int nch, int natm_t,
                             int nks, int nrow, const float* __restrict__ zmax,
                             uint8_t* __restrict__ dst) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (long long)nrow * nks * 2) return;
  const int r = (int)(i % nrow);
  const int u = (int)(i / nrow);  // 8-atom unit: K step u / 2, half u & 1
  const int s = r >> 2, c = r & 3;
  const float sc = tc::pow2_scale(*zmax);
  float f[8];
#pragma unroll
  for (int e = 0; e < 8; ++e) {
    const int a = 8 * u + e;
    f[e] = (s < S && c < nch && a < natm_t) ? (float)zt[(size_t)s * ldz + c * natm_t + a] : 0.f;
  }
  split_store_h(dst + ((size_t)(r / ROWS) * nks + (u >> 1)) * STEP_H + core_off(r % ROWS, 8 * (u & 1)),
                f, sc);
}

// The real views of a type's Mn rows transposed for k_pf_tc: rows = reals k of
// the points (zero past 2 npts), K = atoms (zero past natm_t), from the FP32
// rows sv[a ld_s + k], scaled by pow2_scale(*smax).  One thread = 8 atoms of
// one real.
__global__ void k_presplit_st(const float* __restrict__ sv, long long ld_s, int kr, int natm_t,
                              int nks, int nrow, const float* __restrict__ smax,
                              uint8_t* __restrict__ dst) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (long long)nrow * nks * 2) return;
  const int k = (int)(i % nrow);
  const int u = (int)(i / nrow);
  const float sc = tc::pow2_scale(*smax);
  float f[8];
#pragma unroll
  for (int e = 0; e < 8; ++e) {
    const int a = 8 * u + e;
    f[e] = (k < kr && a < natm_t) ? sv[(size_t)a * ld_s + k] : 0.f;
  }
  split_store_h(dst + ((size_t)(k / ROWS) * nks + (u >> 1)) * STEP_H + core_off(k % ROWS, 8 * (u & 1)),
                f, sc);
}

}  // namespace pctc

template <int NL, bool BM = false>
static int pp_launch(cpstep_ctx* c, dim3 grid, const pctc::PPArgs& pp) {
  using namespace pctc;
  constexpr int BYTES = PPCfg<NL>::BYTES;
  static_assert(BYTES <= 227 * 1024, "shared memory");
  static unsigned long long attr_done = 0;  // per-device attribute, one bit per device
  int dev = 0;
  CPSTEP_CUDA_TRY(cudaGetDevice(&dev));
  const unsigned long long bit = 1ull << (dev & 63);
  if (!(__atomic_load_n(&attr_done, __ATOMIC_ACQUIRE) & bit)) {
    CPSTEP_CUDA_TRY(cudaFuncSetAttribute(k_pp_tc<NL, BM>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         BYTES));
    __atomic_or_fetch(&attr_done, bit, __ATOMIC_RELEASE);
  }
  k_pp_tc<NL, BM><<<grid, PP_NTHR, BYTES, c->stream>>>(pp);
  CPSTEP_LAUNCH_CHECK();
  return CPSTEP_OK;
}

static int hlv_reserve(cpstep_ctx* c, int i, size_t bytes) {
  if (bytes > c->hlv_bytes[i]) {
    graph_drop(c);  // a captured step may hold the old buffer
    cudaFree(c->d_hlv[i]);
    c->d_hlv[i] = nullptr;
    c->hlv_bytes[i] = 0;
    CPSTEP_CUDA_TRY(cudaMalloc(&c->d_hlv[i], bytes));
    c->hlv_bytes[i] = bytes;
  }
  return CPSTEP_OK;
}

// C = alpha overlap(a, b) + beta C for many states (M, N >= 256): both
// operands split once in global memory into their three BF16 levels
// (k_presplit; S's two images, w psi and psi, from one read of psi), the
// product streamed by k_pp_tc<3> (six level products, FP64 folds every 128
// reals), S's diagonal summed in FP64 (k_rowdot).  The in-CTA split of
// k_pc_tc re-reads and re-splits each operand once per tile row or column of
// the output.
static int overlap_stream(cpstep_ctx* c, const double* a, const double* b, int M, int N, int K,
                          const double* w, double alpha, double beta, double* C, int ldc) {
  using namespace pctc;
  const bool same = a == b && M == N;
  const int nsp = pre_nsp(K);
  if (int rc = hlv_reserve(c, 0, pre_bytes(M, K))) return rc;
  if (int rc = hlv_reserve(c, 1, pre_bytes(N, K))) return rc;
  if (same && (size_t)M > c->pdiag_elems) {
    graph_drop(c);
    cudaFree(c->d_pdiag);
    c->d_pdiag = nullptr;
    c->pdiag_elems = 0;
    CPSTEP_CUDA_TRY(cudaMalloc(&c->d_pdiag, sizeof(double) * M));
    c->pdiag_elems = M;
  }
  if (same) {
    k_rowdot<<<M, 256, 0, c->stream>>>(a, K, K, w, c->d_pdiag);
    CPSTEP_LAUNCH_CHECK();
  }
  PreArgs pa{a, K, M, K, nsp, w, 0, c->d_hlv[0], same ? c->d_hlv[1] : nullptr};
  const long long ta = (long long)cdiv(M, ROWS) * nsp * 8 * 32;
  k_presplit<<<(unsigned)((ta + 255) / 256), 256, 0, c->stream>>>(pa);
  CPSTEP_LAUNCH_CHECK();
  if (!same) {
    PreArgs pb{b, K, N, K, nsp, nullptr, 0, c->d_hlv[1], nullptr};
    const long long tb = (long long)cdiv(N, ROWS) * nsp * 8 * 32;
    k_presplit<<<(unsigned)((tb + 255) / 256), 256, 0, c->stream>>>(pb);
    CPSTEP_LAUNCH_CHECK();
  }
  const int tm = cdiv(M, ROWS), tn = cdiv(N, ROWS);
  const int want = std::max(1, c->tune.pc_split * c->num_sms / (tm * tn));
  const int kslab = cdiv(cdiv(K, want), 128) * 128;  // whole fold groups per slab
  const int nsplit = cdiv(K, kslab);
  if (int rc = pc_part_reserve(c, pc_part_need(nsplit, (size_t)M * N))) return rc;
  PPArgs pp{};
  pp.a = c->d_hlv[0];
  pp.b = c->d_hlv[1];
  pp.nsp = nsp;
  pp.M = M;
  pp.N = N;
  pp.K = K;
  pp.kslab = kslab;
  pp.S = M;
  pp.jp = N;
  for (int q = 0; q < 4; ++q) pp.rinv[q] = 1.f;
  pp.cinv = nullptr;
  pp.cstride = 0;
  pp.part = c->d_pc_part;
  pp.err = c->d_dev_err;
  if (int rc = pp_launch<3>(c, dim3(tm, tn, nsplit), pp)) return rc;
  return pc_splitk_reduce_launch(c, nsplit, M, N, alpha, beta, C, ldc, same ? 1 : 0,
                                 same ? c->d_pdiag : nullptr);
}

// Bytes of the EES operand levels (k_presplit_ees_a and the S rows' levels):
// FP16 two-level image of `rows` rows over K reals.
size_t ees_lv_bytes(int rows, int K) {
  using namespace pctc;
  return (size_t)cdiv(rows, ROWS) * (size_t)pre_nsp(K) * STEP_H;
}

// FP16 scale of EES channel c: |w psi| < 4 for states with psi^T psi = 2 I
static float ees_sig(const float* dmax, int c) { return tc::pow2_scale(4.f * dmax[c]); }

// A of the EES sums of ntyp (1 or 2) atom types, split from one read of psi
// into alv[t] (rows c S + s = w psi_s dyp_{t,c}, scale ees_sig(dmax[t], c)).
int ees_tc_presplit_a(cpstep_ctx* c, const double* psi, int ntyp, const float2* const* dyp,
                      int ld_d, const int* nch, const float* const* dmax, uint8_t* const* alv,
                      size_t alv_bytes) {
  using namespace pctc;
  const int S = c->nstates, K = 2 * c->npts, nsp = pre_nsp(K);
  if (ntyp < 1 || ntyp > 2 || (ld_d & 1) || !al16(psi)) return CPSTEP_ERR_ARG;
  PreA pa{};
  pa.psi = psi;
  pa.w = c->d_wpt;
  pa.ntyp = ntyp;
  pa.ld_d = ld_d;
  pa.S = S;
  pa.K = K;
  pa.nsp = nsp;
  for (int t = 0; t < ntyp; ++t) {
    if (nch[t] < 1 || nch[t] > 4 || !al16(dyp[t]) || !al16(alv[t]) ||
        alv_bytes < ees_lv_bytes(nch[t] * S, K))
      return CPSTEP_ERR_ARG;
    pa.dyp[t] = dyp[t];
    pa.nch[t] = nch[t];
    pa.dst[t] = alv[t];
    for (int q = 0; q < 4; ++q) pa.sig[t][q] = q < nch[t] ? ees_sig(dmax[t], q) : 1.f;
  }
  pa.err = c->d_dev_err;
  const long long warps = (long long)cdiv(S, ROWS) * nsp * 8;
  k_presplit_ees_a<<<(unsigned)((warps + 7) / 8), 256, 0, c->stream>>>(pa);  // 8 warps per block
  CPSTEP_LAUNCH_CHECK();
  return CPSTEP_OK;
}

// EES sums of one atom type as the product of two pre-split operands:
// A = w psi dyp_c (rows c S + s, split by ees_tc_presplit_a into alv), B = the
// type's S rows (rows j < jp, FP16 levels at blv, 1 / scale per row at cinv);
// C(s, c jp + j) column-major [nch jp][S].
int ees_tc_sums_pre(cpstep_ctx* c, int nch, const float* dmax, const uint8_t* blv, int jp,
                    const float* cinv, const uint8_t* alv, double* C) {
  using namespace pctc;
  const int S = c->nstates, K = 2 * c->npts, nsp = pre_nsp(K);
  const int M = nch * S;
  if (nch < 1 || nch > 4 || jp < 1 || !al16(blv) || !al16(alv)) return CPSTEP_ERR_ARG;
  const int tm = cdiv(M, ROWS), tn = cdiv(jp, ROWS);
  const int want = std::max(1, c->tune.pc_split * c->num_sms / (tm * tn));
  const int kslab = cdiv(cdiv(K, want), 512) * 512;  // whole fold groups per slab
  const int nsplit = cdiv(K, kslab);
  if (int rc = pc_part_reserve(c, pc_part_need(nsplit, (size_t)M * jp))) return rc;
  PPArgs pp{};
  pp.cstride = 1;
  pp.a = alv;
  pp.b = blv;
  pp.nsp = nsp;
  pp.M = M;
  pp.N = jp;
  pp.K = K;
  pp.kslab = kslab;
  pp.S = S;
  pp.jp = jp;
  for (int q = 0; q < 4; ++q) pp.rinv[q] = q < nch ? 1.f / ees_sig(dmax, q) : 1.f;
  pp.cinv = cinv;
  pp.part = c->d_pc_part;
  pp.err = c->d_dev_err;
  if (int rc = pp_launch<2>(c, dim3(tm, tn, nsplit), pp)) return rc;
  return pc_splitk_reduce_launch(c, nsplit, S, nch * jp, 1.0, 0.0, C, S, 0);
}

// EES psi force of one or two atom types from pre-split operands (k_pf_tc):
// per type Z column-major [S][ldz] (inner index c natm_t + a) and the FP32
// Mn rows sv[a ld_s + k], split into zlv and stlv; F += alpha w sum_t
// (conj(dyp_t) S_t Z_t), F read and written once.
int ees_tc_force_pre(cpstep_ctx* c, int ntyp, const EesForceType* ty, int ld_d, double alpha,
                     double* fpsi, size_t zlv_bytes, size_t stlv_bytes) {
  using namespace pctc;
  const int S = c->nstates, npts = c->npts, kr = 2 * npts;
  const int tm = cdiv(4 * S, ROWS), ntile = cdiv(kr, ROWS);
  if (ntyp < 1 || ntyp > 2 || (ld_d & 1) || !al16(fpsi)) return CPSTEP_ERR_ARG;
  PFArgs pf{};
  pf.ntyp = ntyp;
  for (int t = 0; t < ntyp; ++t) {
    const EesForceType& y = ty[t];
    const int nks = cdiv(y.natm_t, 16);
    if (y.nch < 1 || y.nch > 4 || y.natm_t < 1 || (y.ld_s & 3) || !al16(y.zlv) ||
        !al16(y.stlv) || zlv_bytes < (size_t)tm * nks * STEP_H ||
        stlv_bytes < (size_t)ntile * nks * STEP_H || y.ldz < y.nch * y.natm_t)
      return CPSTEP_ERR_ARG;
    const long long nz = (long long)tm * ROWS * nks * 2, ns = (long long)ntile * ROWS * nks * 2;
    k_presplit_z<<<(unsigned)((nz + 255) / 256), 256, 0, c->stream>>>(
        y.Z, y.ldz, S, y.nch, y.natm_t, nks, tm * ROWS, y.zmax, y.zlv);
    CPSTEP_LAUNCH_CHECK();
    k_presplit_st<<<(unsigned)((ns + 255) / 256), 256, 0, c->stream>>>(
        y.sv, y.ld_s, kr, y.natm_t, nks, ntile * ROWS, y.smax, y.stlv);
    CPSTEP_LAUNCH_CHECK();
    pf.a[t] = y.zlv;
    pf.b[t] = y.stlv;
    pf.nks[t] = nks;
    pf.nch[t] = y.nch;
    pf.zmax[t] = y.zmax;
    pf.smax[t] = y.smax;
    pf.dyp[t] = y.dyp;
  }
  pf.ntile = ntile;
  pf.S = S;
  pf.npts = npts;
  pf.ld_d = ld_d;
  pf.w = c->d_wpt;
  pf.alpha = alpha;
  pf.f = fpsi;
  pf.err = c->d_dev_err;
  static unsigned long long attr_done = 0;  // per-device attribute, one bit per device
  int dev = 0;
  CPSTEP_CUDA_TRY(cudaGetDevice(&dev));
  const unsigned long long bit = 1ull << (dev & 63);
  if (!(__atomic_load_n(&attr_done, __ATOMIC_ACQUIRE) & bit)) {
    CPSTEP_CUDA_TRY(cudaFuncSetAttribute(k_pf_tc, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         PF_BYTES));
    __atomic_or_fetch(&attr_done, bit, __ATOMIC_RELEASE);
  }
  const int gx = std::max(1, std::min(ntile, c->num_sms / tm));
  k_pf_tc<<<dim3(gx, tm), PP_NTHR, PF_BYTES, c->stream>>>(pf);
  CPSTEP_LAUNCH_CHECK();
  return CPSTEP_OK;
}

// Level bytes of the psi force's operands: Z (rows 4 S) and S^T (2 npts reals)
size_t ees_pf_zbytes(int nstates, int natm_t) {
  return (size_t)cdiv(4 * nstates, pctc::ROWS) * cdiv(natm_t, 16) * pctc::STEP_H;
}
size_t ees_pf_stbytes(int npts, int natm_t) {
  return (size_t)cdiv(2 * npts, pctc::ROWS) * cdiv(natm_t, 16) * pctc::STEP_H;
}

// The tensor-core path takes 16-byte aligned operands with even leading
// dimensions and even K (every row segment a whole number of 16-byte pieces),
// and point weights that are powers of two (the context's wpt, 1 or 2), which
// scale the BF16 levels exactly.
bool pc_tc_usable(const cpstep_ctx* c) {
  return c->precision == CPSTEP_PREC_MIXED && c->tc_ok;
}

int pc_overlap_tc_launch(cpstep_ctx* c, const double* a, const double* b, int M, int N, int K,
                         const double* w, double alpha, double beta, double* C, int ldc,
                         bool* used) {
  using namespace pctc;
  *used = false;
  if (!pc_tc_usable(c) || (K & 1) || !al16(a) || !al16(b) || (w && w != c->d_wpt))
    return CPSTEP_OK;
  if (M >= 2 * ROWS && N >= 2 * ROWS) {
    if (int rc = overlap_stream(c, a, b, M, N, K, w, alpha, beta, C, ldc)) return rc;
    *used = true;
    return CPSTEP_OK;
  }
  const bool one = a == b && M == N && M <= ROWS;
  const int tm = cdiv(M, ROWS), tn = cdiv(N, ROWS);
  const int want = std::max(1, c->tune.pc_split * c->num_sms / (tm * tn));
  const int kslab = cdiv(cdiv(K, want), 128) * 128;  // whole TMEM groups per slab
  const int nsplit = cdiv(K, kslab);
  if (int rc = pc_part_reserve(c, pc_part_need(nsplit, (size_t)M * N))) return rc;
  Args p{};
  p.A = a;
  p.B = b;
  p.w = w;
  p.lda = K;
  p.ldb = K;
  p.M = M;
  p.N = N;
  p.K = K;
  p.kslab = kslab;
  p.part = c->d_pc_part;
  p.err = c->d_dev_err;
  p.same = a == b && M == N;
  const dim3 grid(tm, tn, nsplit);
  int rc;
  if (one)
    rc = launch<0, 1, NST_ONE, KC_ONE>(c->stream, grid, p);
  else
    rc = launch<0, 2, NST_TWO, KC_TWO>(c->stream, grid, p);
  if (rc) return rc;
  *used = true;
  return pc_splitk_reduce_launch(c, nsplit, M, N, alpha, beta, C, ldc, p.same);
}

// The back-multiply's matrix, B(i, j) = M(j, i) without its diagonal, is
// split once into the level buffer (offset 0) and shared by all point tiles.
static int backmul_tc(cpstep_ctx* c, const double* Mcm, int ldm, const double* in, int ldi,
                      double* out, int ldo, int nout, int nin, int K, double alpha, double beta,
                      const double* w, const int* psiv_flag, double* psiv_v, double* psiv_no,
                      double rdt, bool* used) {
  using namespace pctc;
  *used = false;
  if (!pc_tc_usable(c) || (K & 1) || (ldm & 1) || (ldi & 1) || !al16(Mcm) || !al16(in))
    return CPSTEP_OK;
  if (psiv_flag && psiv_no != in) return CPSTEP_ERR_ARG;  // psi_no is the input
  // many states: both operands split once and streamed (point tiles on grid y)
  const bool stream = nin >= 2 * ROWS && cdiv(K, ROWS) <= 65535;
  // the PsiV reset rides on k_bm_tc with one column tile, or on the streaming form
  if (psiv_flag && (nin <= 128 ? nout > ROWS : !stream)) return CPSTEP_OK;
  if (int rc = lv_reserve(c, pre_bytes(nout, nin))) return rc;
  if (int rc = presplit(c, Mcm, ldm, nout, nin, nullptr, 1, c->d_lv)) return rc;
  if (stream) {
    const int nsp = pre_nsp(nin);
    if (int rc = hlv_reserve(c, 0, pre_bytes(K, nin))) return rc;
    const long long ta = (long long)cdiv(K, ROWS) * nsp * 8 * 32;
    k_presplit_t<<<(unsigned)((ta + 255) / 256), 256, 0, c->stream>>>(in, ldi, K, nin, nsp,
                                                                       c->d_hlv[0]);
    CPSTEP_LAUNCH_CHECK();
    PPArgs pp{};
    pp.a = c->d_hlv[0];
    pp.b = c->d_lv;
    pp.nsp = nsp;
    pp.M = K;
    pp.N = nout;
    pp.K = nin;
    pp.kslab = cdiv(nin, 128) * 128;
    pp.err = c->d_dev_err;
    pp.in = in;
    pp.m = Mcm;
    pp.w = w;
    pp.out = out;
    pp.ldi = ldi;
    pp.ldm = ldm;
    pp.ldo = ldo;
    pp.alpha = alpha;
    pp.beta = beta;
    pp.psiv_flag = psiv_flag;
    pp.psiv_v = psiv_v;
    pp.rdt = rdt;
    if (int rc = pp_launch<3, true>(c, dim3(cdiv(nout, ROWS), cdiv(K, ROWS), 1), pp)) return rc;
    *used = true;
    return CPSTEP_OK;
  }
  if (nin <= 128) {  // one fold group: the two-CTAs-per-SM kernel
    BMArgs b{};
    b.in = in;
    b.m = Mcm;
    b.pre = c->d_lv;
    b.w = w;
    b.ldi = ldi;
    b.ldm = ldm;
    b.ldo = ldo;
    b.pre_nsp = pre_nsp(nin);
    b.np = K;
    b.nout = nout;
    b.nin = nin;
    b.out = out;
    b.alpha = alpha;
    b.beta = beta;
    b.psiv_flag = psiv_flag;
    b.psiv_v = psiv_v;
    b.psiv_no = psiv_no;
    b.rdt = rdt;
    b.err = c->d_dev_err;
    static unsigned long long attr_done = 0;  // per-device attribute, one bit per device
    int dev = 0;
    CPSTEP_CUDA_TRY(cudaGetDevice(&dev));
    const unsigned long long bit = 1ull << (dev & 63);
    if (!(__atomic_load_n(&attr_done, __ATOMIC_ACQUIRE) & bit)) {
      CPSTEP_CUDA_TRY(
          cudaFuncSetAttribute(k_bm_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, BM_BYTES));
      // the whole unified L1 as shared memory, so that two CTAs fit
      CPSTEP_CUDA_TRY(cudaFuncSetAttribute(k_bm_tc, cudaFuncAttributePreferredSharedMemoryCarveout,
                                           cudaSharedmemCarveoutMaxShared));
      __atomic_or_fetch(&attr_done, bit, __ATOMIC_RELEASE);
    }
    k_bm_tc<<<dim3(cdiv(K, ROWS), cdiv(nout, ROWS)), BM_NTHR, BM_BYTES, c->stream>>>(b);
    CPSTEP_LAUNCH_CHECK();
    *used = true;
    return CPSTEP_OK;
  }
  Args p{};
  p.A = in;
  p.lda = ldi;
  p.B = Mcm;
  p.ldb = ldm;
  p.w = w;
  p.M = K;
  p.N = nout;
  p.K = K;
  p.nin = nin;
  p.out = out;
  p.ldo = ldo;
  p.alpha = alpha;
  p.beta = beta;
  p.err = c->d_dev_err;
  p.pre = c->d_lv;
  p.pre_nsp = pre_nsp(nin);
  if (int rc = launch<1, 1, NST_PRE, KC_PRE>(c->stream, dim3(cdiv(K, ROWS), cdiv(nout, ROWS)), p))
    return rc;
  *used = true;
  return CPSTEP_OK;
}

int pc_backmul_tc_launch(cpstep_ctx* c, const double* Mcm, int ldm, const double* in, int ldi,
                         double* out, int ldo, int nout, int nin, int K, double alpha,
                         double beta, const double* w, bool* used) {
  return backmul_tc(c, Mcm, ldm, in, ldi, out, ldo, nout, nin, K, alpha, beta, w, nullptr,
                    nullptr, nullptr, 0.0, used);
}

// psi = psi_no.T with the PsiV reset in the epilogue (nin <= 128, nout <= 128,
// tensor cores): when *flag, v = (psi_new - psi_old) rdt and psi_no = psi_new.
// *used = false (nothing launched) where the caller must run the reset itself.
int pc_backmul_psiv_tc_launch(cpstep_ctx* c, const double* Tcm, int ldt, double* psi_no,
                              double* psi, int K, int n, const int* flag, double* v, double rdt,
                              bool* used) {
  if (psi_no == psi) {
    *used = false;
    return CPSTEP_OK;
  }
  return backmul_tc(c, Tcm, ldt, psi_no, K, psi, K, n, n, K, 1.0, 0.0, nullptr, flag, v,
                    psi_no, rdt, used);
}
