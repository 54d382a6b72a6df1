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
// at most 128 reals of K (512 in the EES products): it is then read back
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
// An operand that many CTAs share (psi in the EES sums, Z in the EES force,
// T in the back-multiply) is split once, by k_presplit, into its BF16 levels
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
#include "ctx.cuh"
#include "tc_sm100.cuh"

namespace pctc {

constexpr int ROWS = 128;                 // tile rows of A (M) and of B (N)
constexpr int NLV = 3;                    // BF16 levels per element
constexpr int TILE_B = ROWS * 16 * 2;     // one K step, one level, one operand: 4 KB
constexpr int STEP_B = NLV * TILE_B;      // one K step, all levels: 12 KB
constexpr int NW = 512;                   // worker threads (warps 0-15)
constexpr int MMA_WARP = NW / 32;         // warp 16 issues the MMAs
constexpr int NTHR = NW + 32;
constexpr int NSTP_MAX = 5;               // shared-memory stages of a pre-split operand (at most)
constexpr int WBAR = 1;                   // named barrier of the workers
constexpr uint32_t IDESC = tc::idesc_bf16_f32(ROWS, ROWS);
constexpr uint32_t TMEM_COLS = 512;       // two FP32 accumulators + the FP64 tile
constexpr uint32_t TMEM_F64 = 2 * ROWS;   // first column of the FP64 tile

template <int MODE, int NLD, int NST, int KC>
struct Cfg {
  static constexpr int KS = KC / 16;                     // MMA K steps per chunk
  static constexpr int U = KC / 8;                       // 8-element units per row
  // chunks per TMEM group: the hi*hi accumulator holds 128 reals of K for the
  // PairCalc products (S must stay orthonormal to 1e-8) and 512 for the EES
  // sums and psi force (FP32 accumulation over 512 products leaves a relative
  // error near 1e-6 in Z, far inside the energy budget), so their fold of the
  // accumulator into the FP64 tile runs a quarter as often
  static constexpr int NF = (MODE >= 2 ? 512 : 128) / KC;
  static constexpr int RS = KC + 2;                      // row stride of a [128][KC] FP64 stage
  static constexpr int RSP = ROWS + 2;                   // row stride of a [KC][128] FP64 stage
  static constexpr int RSF = KC + 4;                     // [128][KC] FP32 stage
  static constexpr int RSPF = ROWS + 4;                  // [KC][128] FP32 stage
  static constexpr int OPB = KS * STEP_B;                // one operand of one chunk, split
  // operands split in the CTA (CA, CB) or pre-split in global memory (PA, PB)
  static constexpr bool CA = MODE != 2, CB = MODE == 0 || MODE == 2;
  static constexpr bool PA = MODE == 2, PB = MODE == 1 || MODE == 3;
  static constexpr bool PRE = PA || PB;
  // pre-split stages: as deep as shared memory allows (the back-multiply's
  // FP64 [KC][128] stages leave room for 3)
  static constexpr int NSTP = MODE == 1 ? 3 : NSTP_MAX;
  static constexpr int NCONV = (CA ? 1 : 0) + (CB ? 1 : 0);
  static constexpr int RAW0 = ROWS * RS * 8;             // [128][KC] FP64
  static constexpr int WOFF = RAW0 * NLD;                // MODE 0: point weights after the rows
  // one stage: MODE 0 the FP64 rows; MODE 1 in[j][p]; MODE 2 the FP32 S rows
  // and 4 channels' dyp of the chunk's points; MODE 3 the FP32 S rows of the
  // chunk's inner indices and 4 channels' dyp of the tile's points (dyp FP32)
  static constexpr int RAW = MODE == 0   ? WOFF + KC / 2 * 8
                             : MODE == 1 ? KC * RSP * 8
                             : MODE == 2 ? ROWS * RSF * 4 + 4 * (KC / 2) * 8
                                         : KC * RSPF * 4 + 4 * (ROWS / 2) * 8;
  static constexpr int CONV = 2 * NCONV * OPB;           // split operands, two chunk buffers
  static constexpr int PREB = PRE ? NSTP * OPB : 0;      // pre-split operand stages
  static constexpr int BYTES = 1024 + CONV + PREB + NST * RAW;  // + alignment slack
  static_assert(KC % 16 == 0 && 128 % KC == 0, "chunk");
  static_assert(RAW % 16 == 0 && OPB % 1024 == 0, "stage alignment");
  static_assert(ROWS * U * (MODE == 0 ? NLD : 1) == NW, "one 8-element unit per worker");
  static_assert(ROWS * (KC / 2) % NW == 0 && KC * (ROWS / 2) % NW == 0 &&
                    KC * (ROWS / 4) % NW == 0,
                "copy mapping");
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
  // EES (MODE 2: forward sums, MODE 3: psi force), one atom type:
  //   sv: S rows of the type, row j at sv + j ld_s (floats, complex pairs per
  //       point); MODE 2 pairs j = v natm_t + a (v = Mn, d/dx, d/dy, d/dz),
  //       MODE 3 rows a < natm_t (Mn)
  //   dyp: the type's nch channel projectors (FP32), channel c at dyp + c ld_d
  //        (ld_d even: 16-byte rows)
  //   MODE 2: B-tile rows c jt + jj (c < nch, jj < jt) = channel c x pair
  //           t jt + jj, jp pairs; output column c jp + j
  //   MODE 3: inner index j = c natm_t + a (nin = nch natm_t)
  const float* sv;
  long long ld_s;
  const float2* dyp;
  int ld_d;
  int nch, jt, jp, natm_t;
  double alpha, beta;
  // pre-split operand (MODE 2: A = w psi; MODE 1: B = M^T without its
  // diagonal; MODE 3: B = Z^T): [row tile][K step][level][4 KB], pre_nsp
  // K steps per row tile
  const uint8_t* pre;
  int pre_nsp;
  int* err;
};

// byte offset of (row r, k) in one K-step tile (k < 16)
__host__ __device__ __forceinline__ int core_off(int r, int k) {
  return (r >> 3) * 256 + (k >> 3) * 128 + (r & 7) * 16 + (k & 7) * 2;
}

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
  to_f32(x, ws, f);
  split_store(a.dst + ((size_t)rt * a.nsp + s) * STEP_B + core_off(rl, 8 * kh), f);
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
  if (MODE == 0 || MODE == 2) {
    r0 = blockIdx.x * ROWS;
    c0 = blockIdx.y * (MODE == 2 ? p.jt : ROWS);  // MODE 2: first pair of the B tile
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
            p.pre + ((size_t)prow * p.pre_nsp + (size_t)((kbeg + c * KC) >> 4)) * STEP_B;
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
            const uint64_t da = tc::smem_desc_kmajor(a0 + s * STEP_B + LA[t] * TILE_B, 128, 256);
            const uint64_t db = tc::smem_desc_kmajor(b0 + s * STEP_B + LB[t] * TILE_B, 128, 256);
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
      } else if (MODE == 2) {
        // S rows of pairs c0 .. c0 + jt, KC reals (FP32), and dyp of the chunk's points
        float* fs = reinterpret_cast<float*>(ra);
        for (int q = tid; q < p.jt * (KC / 4); q += NW) {
          const int jj = q / (KC / 4), pc = q % (KC / 4);
          const int j = c0 + jj, k = k0 + 4 * pc;
          const bool ok = j < p.jp && k < kend;  // kend even, rows padded to 4 floats
          const float* g = ok ? p.sv + (size_t)j * p.ld_s + k : p.sv;
          tc::cp16(fs + jj * C::RSF + 4 * pc, g, ok ? 16 : 0);
        }
        float2* dd = reinterpret_cast<float2*>(fs + ROWS * C::RSF);
        for (int q = tid; q < p.nch * (KC / 4); q += NW) {  // two points per copy
          const int c = q / (KC / 4), e = 2 * (q % (KC / 4));
          const int pt = (k0 >> 1) + e;
          const int nb = 2 * pt + 2 < kend ? 16 : (2 * pt < kend ? 8 : 0);
          tc::cp16(dd + c * (KC / 2) + e, nb ? p.dyp + (size_t)c * p.ld_d + pt : p.dyp, nb);
        }
      } else if (MODE == 3) {
        // S rows (Mn) of the chunk's inner indices j = c natm_t + a over the
        // tile's 64 points, and the channels' dyp over the same points
        float* fs = reinterpret_cast<float*>(ra);
#pragma unroll
        for (int it = 0; it < KC * (ROWS / 4) / NW; ++it) {
          const int q = tid + NW * it;
          const int jj = q / (ROWS / 4), pc = q % (ROWS / 4);
          const int j = k0 + jj, pr = r0 + 4 * pc;  // reals
          const bool ok = j < kend && pr < p.M;      // M reals, rows padded to 4 floats
          const int a = ok ? j % p.natm_t : 0;
          const float* g = ok ? p.sv + (size_t)a * p.ld_s + pr : p.sv;
          tc::cp16(fs + jj * C::RSPF + 4 * pc, g, ok ? 16 : 0);
        }
        float2* dd = reinterpret_cast<float2*>(fs + KC * C::RSPF);
        for (int q = tid; q < p.nch * (ROWS / 4); q += NW) {  // two points per copy
          const int c = q / (ROWS / 4), e = 2 * (q % (ROWS / 4));
          const int pt = (r0 >> 1) + e;
          const int nb = 2 * pt + 2 < p.M ? 16 : (2 * pt < p.M ? 8 : 0);
          tc::cp16(dd + c * (ROWS / 2) + e, nb ? p.dyp + (size_t)c * p.ld_d + pt : p.dyp, nb);
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
      const int op = (MODE == 0 && NLD == 2) ? (tid >> 8) : (MODE == 2 ? 1 : 0);
      const int q = (MODE == 0 && NLD == 2) ? (tid & 255) : tid;
      const int r = (q & 7) + 8 * ((q >> 3) / U), u = (q >> 3) % U;
      const int off = (u >> 1) * STEP_B + core_off(r, (u & 1) * 8);
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
      // EES operands in FP32 (S is FP32): conj(dyp) S, one rounding per product
      if (MODE == 3) {  // A[p][j] = (conj(dyp_c) S_a)(point r / 2), re or im
        const float* fs = reinterpret_cast<const float*>(ra);
        const float2* dd = reinterpret_cast<const float2*>(fs + KC * C::RSPF);
        const int pl = r >> 1;
#pragma unroll
        for (int e = 0; e < 8; ++e) {
          const int j = k0 + 8 * u + e;
          const int c = min(j / p.natm_t, 3);
          const float2 sa = *reinterpret_cast<const float2*>(fs + (8 * u + e) * C::RSPF + 2 * pl);
          const float2 d = dd[c * (ROWS / 2) + pl];
          f[e] = (r & 1) ? fmaf(d.x, sa.y, -d.y * sa.x) : fmaf(d.x, sa.x, d.y * sa.y);
        }
        split_store(dA, f);
        return;
      }
      if (MODE == 2) {  // B row r = channel c, pair jj: conj(dyp_c) S_pair
        const float* fs = reinterpret_cast<const float*>(ra);
        const float2* dd = reinterpret_cast<const float2*>(fs + ROWS * C::RSF);
        const int c = r / p.jt, jj = r - c * p.jt;
        const bool ok = c < p.nch;
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          const float2 sa =
              ok ? *reinterpret_cast<const float2*>(fs + jj * C::RSF + 8 * u + 2 * e)
                 : make_float2(0.f, 0.f);
          const float2 d = ok ? dd[c * (KC / 2) + 4 * u + e] : make_float2(0.f, 0.f);
          f[2 * e] = fmaf(d.x, sa.x, d.y * sa.y);
          f[2 * e + 1] = fmaf(d.x, sa.y, -d.y * sa.x);
        }
        split_store(dB, f);
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
    const double sc = (MODE == 1 || MODE == 3) && r0 + rl < p.M
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
        } else if (MODE == 2) {  // tile column cb + e = channel ch, pair c0 + jj -> ch jp + pair
          const int r = r0 + rl;
          const int ch = (cb + e) / p.jt, j = c0 + (cb + e) - ch * p.jt;
          if (r < p.M && ch < p.nch && j < p.jp)
            p.part[(size_t)blockIdx.z * p.M * p.N + (size_t)(ch * p.jp + j) * p.M + r] = acc;
        } else {
          accs[e8] = acc;
        }
      }
      if (MODE == 1 || MODE == 3) {
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
  PreArgs a{src, ldr, rows, K, pre_nsp(K), w, zero_diag, dst};
  const long long threads = (long long)cdiv(rows, ROWS) * a.nsp * 8 * 32;
  k_presplit<<<(unsigned)((threads + 255) / 256), 256, 0, c->stream>>>(a);
  CPSTEP_LAUNCH_CHECK();
  return CPSTEP_OK;
}

}  // namespace pctc

// BF16 levels of w psi for the EES sums (offset 0 of the level buffer), with
// room after them for a Z of up to nin_max inner indices (ees_tc_force).
int ees_tc_presplit(cpstep_ctx* c, const double* psi, int nin_max) {
  using namespace pctc;
  const int S = c->nstates, K = 2 * c->npts;
  if (!al16(psi) || nin_max < 1) return CPSTEP_ERR_ARG;
  if (int rc = lv_reserve(c, pre_bytes(S, K) + pre_bytes(S, nin_max))) return rc;
  return presplit(c, psi, K, S, K, c->d_wpt, 0, c->d_lv);
}

// EES sums of one atom type (MODE 2): C(s, ch jp + j) = sum_p wpt Re(conj psi_s
// conj(dyp_ch) S_j), j < jp pairs; C column-major [nch jp][ldc], alpha = 1.
// Takes psi's levels from ees_tc_presplit.
int ees_tc_sums(cpstep_ctx* c, const float* sv, long long ld_s, const float2* dyp, int ld_d,
                int nch, int jp, double* C, int ldc) {
  using namespace pctc;
  const int S = c->nstates, K = 2 * c->npts;
  if (nch < 1 || nch > 4 || (ld_s & 3) || (ld_d & 1) || !al16(sv) || !al16(dyp) ||
      c->lv_bytes < pre_bytes(S, K))
    return CPSTEP_ERR_ARG;
  const int jt = ROWS / nch;
  const int tm = cdiv(S, ROWS), tn = cdiv(jp, jt);
  const int want = std::max(1, c->tune.pc_split * c->num_sms / (tm * tn));
  const int kslab = cdiv(cdiv(K, want), 128) * 128;
  const int nsplit = cdiv(K, kslab);
  const int N = nch * jp;
  if (int rc = pc_part_reserve(c, (size_t)nsplit * S * N)) return rc;
  Args p{};
  p.lda = K;
  p.M = S;
  p.N = N;
  p.K = K;
  p.kslab = kslab;
  p.part = c->d_pc_part;
  p.err = c->d_dev_err;
  p.sv = sv;
  p.ld_s = ld_s;
  p.dyp = dyp;
  p.ld_d = ld_d;
  p.nch = nch;
  p.jt = jt;
  p.jp = jp;
  p.pre = c->d_lv;
  p.pre_nsp = pre_nsp(K);
  if (int rc = launch<2, 1, NST_PRE, KC_PRE>(c->stream, dim3(tm, tn, nsplit), p)) return rc;
  return pc_splitk_reduce_launch(c, nsplit, S, N, 1.0, 0.0, C, ldc, 0);
}

// EES psi force of one atom type (MODE 3): fpsi_s(p) += alpha wpt(p) sum_j
// Z(j, s) (conj(dyp_c) S_a)(p), j = c natm_t + a; Z column-major [S][ldz].
// Z's levels go after psi's (room reserved by ees_tc_presplit).
int ees_tc_force(cpstep_ctx* c, const float* sv, long long ld_s, const float2* dyp, int ld_d,
                 int nch, int natm_t, const double* Z, int ldz, double alpha, double* fpsi) {
  using namespace pctc;
  const int S = c->nstates, K = 2 * c->npts, nin = nch * natm_t;
  if (nch < 1 || nch > 4 || (ld_s & 3) || (ld_d & 1) || (ldz & 1) || !al16(sv) || !al16(Z) ||
      !al16(dyp) || c->lv_bytes < pre_bytes(S, K) + pre_bytes(S, nin))
    return CPSTEP_ERR_ARG;
  uint8_t* zl = c->d_lv + pre_bytes(S, K);
  if (int rc = presplit(c, Z, ldz, S, nin, nullptr, 0, zl)) return rc;
  Args p{};
  p.w = c->d_wpt;
  p.M = K;
  p.N = S;
  p.K = K;
  p.nin = nin;
  p.out = fpsi;
  p.ldo = K;
  p.alpha = alpha;
  p.beta = 1.0;
  p.err = c->d_dev_err;
  p.sv = sv;
  p.ld_s = ld_s;
  p.dyp = dyp;
  p.ld_d = ld_d;
  p.nch = nch;
  p.natm_t = natm_t;
  p.pre = zl;
  p.pre_nsp = pre_nsp(nin);
  return launch<3, 1, NST_PRE, KC_PRE>(c->stream, dim3(cdiv(K, ROWS), cdiv(S, ROWS)), p);
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
  const bool one = a == b && M == N && M <= ROWS;
  const int tm = cdiv(M, ROWS), tn = cdiv(N, ROWS);
  const int want = std::max(1, c->tune.pc_split * c->num_sms / (tm * tn));
  const int kslab = cdiv(cdiv(K, want), 128) * 128;  // whole TMEM groups per slab
  const int nsplit = cdiv(K, kslab);
  if (int rc = pc_part_reserve(c, (size_t)nsplit * M * N)) return rc;
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
int pc_backmul_tc_launch(cpstep_ctx* c, const double* Mcm, int ldm, const double* in, int ldi,
                         double* out, int ldo, int nout, int nin, int K, double alpha,
                         double beta, const double* w, bool* used) {
  using namespace pctc;
  *used = false;
  if (!pc_tc_usable(c) || (K & 1) || (ldm & 1) || (ldi & 1) || !al16(Mcm) || !al16(in))
    return CPSTEP_OK;
  if (int rc = lv_reserve(c, pre_bytes(nout, nin))) return rc;
  if (int rc = presplit(c, Mcm, ldm, nout, nin, nullptr, 1, c->d_lv)) return rc;
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
