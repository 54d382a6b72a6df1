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
// accumulated by tcgen05.mma (kind::f16, BF16 in, FP32 accumulator in TMEM),
// smallest terms first.  The FP32 accumulator holds at most 128 reals of K:
// it is then read back (tcgen05.ld) and added into FP64 registers, so the sums
// over those groups, over the split-K slabs and the epilogue terms are FP64.
//
// One CTA = one 128 x 128 output tile (M = N = 128 MMA) and one K range,
// 512 threads, one CTA per SM:
//   * cp.async brings the FP64 operand chunks (KC reals) into NST
//     shared-memory stages (one operand when A and B are the same rows:
//     S = psi^T psi);
//   * all threads split a stage into BF16 levels in the K-major no-swizzle
//     core-matrix layout (8 rows x 16 bytes per core matrix; the two 8-element
//     K halves of a 16-wide K step 128 bytes apart, 8-row groups 256 bytes
//     apart), applying the per-point weight (a power of two: exact) on the way;
//   * thread 0 issues the 6 MMAs per K step of the chunk into one of two TMEM
//     accumulator pairs (hi*hi and the five small products apart) and
//     commits them to an mbarrier;
//   * while they run, all threads start the copies of a later chunk and,
//     after every NF chunks, fold the accumulator into FP64.
// Every mbarrier wait is bounded (1 s): on a time-out the CTA records an error
// bit in *err, drains its copies, waits (bounded) for its MMAs, releases TMEM
// and returns without writing its tile.
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
constexpr int NTHR = 512;
constexpr uint32_t IDESC = tc::idesc_bf16_f32(ROWS, ROWS);
constexpr uint32_t TMEM_COLS = 512;       // two groups x (hi*hi, corrections) FP32 accumulators

template <int MODE, int NLD, int NST, int KC>
struct Cfg {
  static constexpr int KS = KC / 16;                     // MMA K steps per chunk
  static constexpr int U = KC / 8;                       // 8-element units per row
  static constexpr int NF = 128 / KC;                    // chunks per TMEM group
  static constexpr int RS = KC + 2;                      // row stride of a [128][KC] stage
  static constexpr int RSP = ROWS + 2;                   // row stride of a [KC][128] stage
  static constexpr int LVB = KS * TILE_B;                // one level of one operand
  static constexpr int OPB = NLV * LVB;                  // one operand of one chunk
  // EES (MODE 2, 3): FP32 complex S rows (stride RSF / RSPF floats) and the
  // channels' projector values dyp (double2) staged beside them
  static constexpr int RSF = KC + 4;                     // [rows][KC] floats
  static constexpr int RSPF = ROWS + 4;                  // [KC][128] floats
  static constexpr int DYP2 = 4 * (KC / 2) * 16;         // MODE 2: 4 channels x KC/2 points
  static constexpr int DYP3 = 4 * (ROWS / 2) * 16;       // MODE 3: 4 channels x 64 points
  static constexpr int RAW_A = (MODE == 0 || MODE == 2) ? ROWS * RS * 8
                               : MODE == 1 ? KC * RSP * 8 : KC * RSPF * 4 + DYP3;
  static constexpr int RAW_B = MODE == 2 ? ROWS * RSF * 4 + DYP2 : ROWS * RS * 8;
  static constexpr int WST = (MODE == 0 || MODE == 2) ? KC / 2 * 8 : 0;  // point weights
  static constexpr int WOFF = RAW_A + (NLD == 2 ? RAW_B : 0);      // weights in a stage
  static constexpr int RAW = WOFF + WST;                            // one stage
  static constexpr int BF = 2 * 2 * OPB;                 // two chunk buffers, A and B
  static constexpr int BYTES = 1024 + BF + NST * RAW;    // + alignment slack
  static_assert(KC % 16 == 0 && 128 % KC == 0, "chunk");
  // conversion: one 8-element unit per thread (NLD = 2: threads < 256 take A)
  static_assert(ROWS * U * NLD == NTHR, "thread mapping");
  static_assert(ROWS * (KC / 2) % NTHR == 0 && KC * (ROWS / 2) % NTHR == 0, "copy mapping");
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
  //   dyp: the type's nch channel projectors, channel c at dyp + c ld_d
  //   MODE 2: B-tile rows c jt + jj (c < nch, jj < jt) = channel c x pair
  //           t jt + jj, jp pairs; output column c jp + j
  //   MODE 3: inner index j = c natm_t + a (nin = nch natm_t)
  const float* sv;
  long long ld_s;
  const double2* dyp;
  int ld_d;
  int nch, jt, jp, natm_t;
  double alpha, beta;
  int* err;
};

// byte offset of (row r, k) in one K-step tile (k < 16)
__device__ __forceinline__ int core_off(int r, int k) {
  return (r >> 3) * 256 + (k >> 3) * 128 + (r & 7) * 16 + (k & 7) * 2;
}

template <int MODE, int NLD, int NST, int KC>
__global__ void __launch_bounds__(NTHR, 1) k_pc_tc(const Args p) {
  using C = Cfg<MODE, NLD, NST, KC>;
  constexpr int KS = C::KS, U = C::U, NF = C::NF, RS = C::RS, RSP = C::RSP;
  constexpr bool DIAG = MODE == 0;
  extern __shared__ uint8_t dsm[];
  __shared__ uint64_t bar[2];
  __shared__ uint32_t tslot;
  __shared__ double diag_s[DIAG ? ROWS : 1];
  const uint32_t s0 = tc::smem_u32(dsm);
  uint8_t* base = dsm + (((s0 + 1023u) & ~1023u) - s0);
  const uint32_t bf_s = tc::smem_u32(base);   // [2 buffers][A,B][level][KS][4 KB]
  double* raw = reinterpret_cast<double*>(base + C::BF);
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
  double dacc = 0.0;

  if (warp == 0) tc::tmem_alloc(&tslot, TMEM_COLS);
  if (tid == 0) {
    tc::mbar_init(&bar[0], 1);
    tc::mbar_init(&bar[1], 1);
    tc::fence_mbar_init();
  }
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tbase = tslot;

  // ---- copies of chunk ch into stage st
  auto load = [&](int ch, int st) {
    const int k0 = kbeg + ch * KC;
    double* ra = raw + (size_t)st * (C::RAW / 8);
    if (MODE == 0 || MODE == 2) {
#pragma unroll
      for (int op = 0; op < (MODE == 2 ? 1 : NLD); ++op) {
        const double* src = op == 0 ? p.A : p.B;
        const int ld = op == 0 ? p.lda : p.ldb;
        const int rr0 = op == 0 ? r0 : c0, nr = op == 0 ? p.M : p.N;
        double* dst = ra + op * (C::RAW_A / 8);
        if (op == 0 && p.w && tid < KC / 4) {  // weights of points k0/2 .. (k0 + KC)/2
          const int pt = (k0 >> 1) + 2 * tid;
          const int nb = 2 * pt + 2 < kend ? 16 : (2 * pt < kend ? 8 : 0);
          tc::cp16(ra + C::WOFF / 8 + 2 * tid, nb ? p.w + pt : p.w, nb);
        }
#pragma unroll
        for (int it = 0; it < ROWS * (KC / 2) / NTHR; ++it) {
          const int q = tid + NTHR * it;
          const int r = q / (KC / 2), pc = q % (KC / 2);
          const int k = k0 + 2 * pc;
          const bool ok = rr0 + r < nr && k < kend;  // kend even: the pair is inside
          const double* g = ok ? src + (size_t)(rr0 + r) * ld + k : src;
          tc::cp16(dst + r * RS + 2 * pc, g, ok ? 16 : 0);
        }
      }
      if (MODE == 2) {
        // B: S rows of pairs c0 .. c0 + jt, KC reals (FP32), and dyp of the chunk's points
        float* fs = reinterpret_cast<float*>(ra + C::RAW_A / 8);
        for (int q = tid; q < p.jt * (KC / 4); q += NTHR) {
          const int jj = q / (KC / 4), pc = q % (KC / 4);
          const int j = c0 + jj, k = k0 + 4 * pc;
          const bool ok = j < p.jp && k < kend;  // kend even, rows padded to 4 floats
          const float* g = ok ? p.sv + (size_t)j * p.ld_s + k : p.sv;
          tc::cp16(fs + jj * C::RSF + 4 * pc, g, ok ? 16 : 0);
        }
        double2* dd = reinterpret_cast<double2*>(fs + ROWS * C::RSF);
        for (int q = tid; q < p.nch * (KC / 2); q += NTHR) {
          const int c = q / (KC / 2), e = q % (KC / 2);
          const int pt = (k0 >> 1) + e;
          const bool ok = 2 * pt < kend;
          tc::cp16(dd + c * (KC / 2) + e, ok ? p.dyp + (size_t)c * p.ld_d + pt : p.dyp,
                   ok ? 16 : 0);
        }
      }
    } else if (MODE == 3) {
      // A: S rows (Mn) of the chunk's inner indices j = c natm_t + a over the
      // tile's 64 points, and the channels' dyp over the same points
      float* fs = reinterpret_cast<float*>(ra);
#pragma unroll
      for (int it = 0; it < KC * (ROWS / 4) / NTHR; ++it) {
        const int q = tid + NTHR * it;
        const int jj = q / (ROWS / 4), pc = q % (ROWS / 4);
        const int j = k0 + jj, pr = r0 + 4 * pc;  // reals
        const bool ok = j < kend && pr < p.M;      // M reals, rows padded to 4 floats
        const int a = ok ? j % p.natm_t : 0;
        const float* g = ok ? p.sv + (size_t)a * p.ld_s + pr : p.sv;
        tc::cp16(fs + jj * C::RSPF + 4 * pc, g, ok ? 16 : 0);
      }
      double2* dd = reinterpret_cast<double2*>(fs + KC * C::RSPF);
      for (int q = tid; q < p.nch * (ROWS / 2); q += NTHR) {
        const int c = q / (ROWS / 2), e = q % (ROWS / 2);
        const int pt = (r0 >> 1) + e;
        const bool ok = 2 * pt < p.M;
        tc::cp16(dd + c * (ROWS / 2) + e, ok ? p.dyp + (size_t)c * p.ld_d + pt : p.dyp,
                 ok ? 16 : 0);
      }
      // B: M(j, i) = Mcm[j + i ldm], rows i = c0 .. c0 + 128, j pairs
      double* rb = ra + C::RAW_A / 8;
#pragma unroll
      for (int it = 0; it < ROWS * (KC / 2) / NTHR; ++it) {
        const int q = tid + NTHR * it;
        const int r = q / (KC / 2), pc = q % (KC / 2);
        const int i = c0 + r, j = k0 + 2 * pc;
        const int nb = (i < p.N && j < kend) ? (j + 1 < kend ? 16 : 8) : 0;
        const double* g = nb ? p.B + (size_t)i * p.ldb + j : p.B;
        tc::cp16(rb + r * RS + 2 * pc, g, nb);
      }
    } else {
      // A: in[j][p] rows j = k0 .. k0 + KC, 128 points from r0
#pragma unroll
      for (int it = 0; it < KC * (ROWS / 2) / NTHR; ++it) {
        const int q = tid + NTHR * it;
        const int jj = q / (ROWS / 2), pc = q % (ROWS / 2);
        const int j = k0 + jj, pt = r0 + 2 * pc;
        const bool ok = j < kend && pt < p.M;  // M (reals) even
        const double* g = ok ? p.A + (size_t)j * p.lda + pt : p.A;
        tc::cp16(ra + jj * RSP + 2 * pc, g, ok ? 16 : 0);
      }
      // B: M(j, i) = Mcm[j + i ldm], rows i = c0 .. c0 + 128, j pairs
      double* rb = ra + C::RAW_A / 8;
#pragma unroll
      for (int it = 0; it < ROWS * (KC / 2) / NTHR; ++it) {
        const int q = tid + NTHR * it;
        const int r = q / (KC / 2), pc = q % (KC / 2);
        const int i = c0 + r, j = k0 + 2 * pc;
        const int nb = (i < p.N && j < kend) ? (j + 1 < kend ? 16 : 8) : 0;
        const double* g = nb ? p.B + (size_t)i * p.ldb + j : p.B;
        tc::cp16(rb + r * RS + 2 * pc, g, nb);
      }
    }
  };

  // ---- 8 FP64 values -> three BF16 levels stored at level offsets
  auto put = [&](uint8_t* dst, int off, const double (&x)[8], const float (&ws)[4]) {
    uint32_t lv[NLV][4];
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      uint32_t a[NLV], b[NLV];
      tc::split3(x[2 * e], a);
      tc::split3(x[2 * e + 1], b);
#pragma unroll
      for (int v = 0; v < NLV; ++v) {
        const float fa = __uint_as_float(a[v]) * ws[e], fb = __uint_as_float(b[v]) * ws[e];
        lv[v][e] = tc::pack_bf16x2(__float_as_uint(fa), __float_as_uint(fb));
      }
    }
#pragma unroll
    for (int v = 0; v < NLV; ++v)
      *reinterpret_cast<uint4*>(dst + v * C::LVB + off) =
          make_uint4(lv[v][0], lv[v][1], lv[v][2], lv[v][3]);
  };

  // ---- stage st (chunk ch) -> BF16 buffer buf: one 8-element unit per
  // thread; NLD = 1 puts it into A (weighted) and B, NLD = 2 gives A to the
  // first 256 threads and B to the rest
  auto convert = [&](int ch, int st, int buf) {
    const int k0 = kbeg + ch * KC;
    const double* ra = raw + (size_t)st * (C::RAW / 8);
    const int op = NLD == 2 ? (tid >> 8) : 0;
    const int q = NLD == 2 ? (tid & 255) : tid;
    const int r = (q & 7) + 8 * ((q >> 3) / U), u = (q >> 3) % U;
    const int off = (u >> 1) * TILE_B + core_off(r, (u & 1) * 8);
    uint8_t* dA = base + (size_t)(buf * 2 + 0) * C::OPB;
    uint8_t* dB = base + (size_t)(buf * 2 + 1) * C::OPB;
    const float one[4] = {1.f, 1.f, 1.f, 1.f};
    double x[8];
    if (MODE == 1 && op == 0) {  // A[p][j] = in[j][p] from the [KC][128] stage
#pragma unroll
      for (int e = 0; e < 8; ++e) x[e] = ra[(8 * u + e) * RSP + r];
      put(dA, off, x, one);
      return;
    }
    if (MODE == 3 && op == 0) {  // A[p][j] = (conj(dyp_c) S_a)(point r / 2), re or im
      const float* fs = reinterpret_cast<const float*>(ra);
      const double2* dd = reinterpret_cast<const double2*>(fs + KC * C::RSPF);
      const int pl = r >> 1;
#pragma unroll
      for (int e = 0; e < 8; ++e) {
        const int j = k0 + 8 * u + e;
        const int c = min(j / p.natm_t, 3);
        const float2 sa = *reinterpret_cast<const float2*>(fs + (8 * u + e) * C::RSPF + 2 * pl);
        const double2 d = dd[c * (ROWS / 2) + pl];
        x[e] = (r & 1) ? d.x * (double)sa.y - d.y * (double)sa.x
                       : d.x * (double)sa.x + d.y * (double)sa.y;
      }
      put(dA, off, x, one);
      return;
    }
    if (MODE == 2 && op == 1) {  // B row r = channel c, pair jj: conj(dyp_c) S_pair
      const float* fs = reinterpret_cast<const float*>(ra + C::RAW_A / 8);
      const double2* dd = reinterpret_cast<const double2*>(fs + ROWS * C::RSF);
      const int c = r / p.jt, jj = r - c * p.jt;
      const bool ok = c < p.nch;
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const float2 sa =
            ok ? *reinterpret_cast<const float2*>(fs + jj * C::RSF + 8 * u + 2 * e)
               : make_float2(0.f, 0.f);
        const double2 d = ok ? dd[c * (KC / 2) + 4 * u + e] : make_double2(0.0, 0.0);
        x[2 * e] = d.x * (double)sa.x + d.y * (double)sa.y;
        x[2 * e + 1] = d.x * (double)sa.y - d.y * (double)sa.x;
      }
      put(dB, off, x, one);
      return;
    }
    const double2* s2 =
        reinterpret_cast<const double2*>(ra + op * (C::RAW_A / 8) + r * RS + 8 * u);
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      const double2 v = s2[e];
      x[2 * e] = v.x;
      x[2 * e + 1] = v.y;
    }
    if (MODE == 1 || MODE == 3) {  // B[i][j] = M(j, i); MODE 1: diagonal left to the epilogue
      if (MODE == 1) {
        const int d = (c0 + r) - (k0 + 8 * u);
#pragma unroll
        for (int e = 0; e < 8; ++e)
          if (e == d) x[e] = 0.0;
      }
      put(dB, off, x, one);
      return;
    }
    if (op == 1) {
      put(dB, off, x, one);
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
    put(dA, off, x, ws);
    if (NLD == 1) put(dB, off, x, one);
  };

  // ---- the MMAs of chunk ch (thread 0), smallest level products first
  // hi*hi goes to its own accumulator (columns +128), so the FP32 rounding of
  // the sum of the small terms is relative to their own size
  auto issue = [&](int ch) {
    const int buf = ch & 1;
    const uint32_t td = tbase + (uint32_t)(((ch / NF) & 1) * 2 * ROWS);
    const uint32_t a0 = bf_s + (uint32_t)((buf * 2 + 0) * C::OPB);
    const uint32_t b0 = bf_s + (uint32_t)((buf * 2 + 1) * C::OPB);
    constexpr int PA[6] = {2, 0, 1, 1, 0, 0};
    constexpr int PB[6] = {0, 2, 1, 0, 1, 0};
#pragma unroll
    for (int s = 0; s < KS; ++s) {
#pragma unroll
      for (int t = 0; t < 6; ++t) {
        const uint64_t da = tc::smem_desc_kmajor(a0 + PA[t] * C::LVB + s * TILE_B, 128, 256);
        const uint64_t db = tc::smem_desc_kmajor(b0 + PB[t] * C::LVB + s * TILE_B, 128, 256);
        const uint32_t accum = (ch % NF == 0 && s == 0 && (t == 0 || t == 5)) ? 0u : 1u;
        tc::mma_bf16(t == 5 ? td + ROWS : td, da, db, IDESC, accum);
      }
    }
    tc::commit(&bar[buf]);
  };

  // ---- TMEM accumulators of group g -> FP64 registers (warp w: lanes
  // 32 (w % 4) .., columns 32 (w / 4) ..)
  double acc[32];
#pragma unroll
  for (int e = 0; e < 32; ++e) acc[e] = 0.0;
  auto flush = [&](int g) {
    tc::fence_after_sync();
    const uint32_t ta = tbase + ((uint32_t)(32 * (warp & 3)) << 16) +
                        (uint32_t)((g & 1) * 2 * ROWS + 32 * (warp >> 2));
#pragma unroll
    for (int hh = 0; hh < 2; ++hh) {
      float v[32];
      tc::tmem_ld32(ta + hh * ROWS, v);
#pragma unroll
      for (int e = 0; e < 32; ++e) acc[e] += (double)v[e];
    }
    tc::fence_before_sync();
  };
  // MMAs up to chunk ch complete; warp-uniform (tcgen05.ld is warp-collective)
  auto wait_chunk = [&](int ch) -> bool {
    return __all_sync(0xffffffffu, tc::mbar_wait(&bar[ch & 1], (ch >> 1) & 1));
  };

#pragma unroll
  for (int ch = 0; ch < NST - 1; ++ch) {
    if (ch < nch) load(ch, ch);
    tc::cp_commit();
  }
  int bad = 0, issued = 0;
  for (int ch = 0; ch < nch; ++ch) {
    tc::cp_wait<NST - 2>();
    if (__syncthreads_or(bad)) {
      bad = 1;
      break;
    }
    convert(ch, ch % NST, ch & 1);
    tc::fence_async_shared();
    tc::fence_before_sync();
    __syncthreads();
    if (tid == 0) {
      tc::fence_after_sync();
      issue(ch);
    }
    issued = ch + 1;
    if (ch + NST - 1 < nch) load(ch + NST - 1, (ch + NST - 1) % NST);
    tc::cp_commit();
    if (ch >= 1) {  // frees BF16 buffer (ch + 1) & 1; folds a finished group
      if (!wait_chunk(ch - 1))
        bad = 1;
      else if ((ch - 1) % NF == NF - 1)
        flush((ch - 1) / NF);
    }
  }
  bad = __syncthreads_or(bad);
  if (!bad && nch > 0) {
    if (wait_chunk(nch - 1))
      flush((nch - 1) / NF);
    else
      bad = 1;
  }
  bad = __syncthreads_or(bad);
  if (bad && issued > 0 && warp == 0)  // nothing may still write TMEM when it is released
    wait_chunk(issued - 1);
  tc::cp_wait<0>();
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) {
    tc::fence_after_sync();
    tc::tmem_free(tbase, TMEM_COLS);
  }
  if (bad) {
    if (tid == 0) atomicOr(p.err, 1);
    return;
  }
  if (DIAG && same) {  // the U units of row r sit in lanes l, l + 8, ... (same warp)
    double d = dacc;
#pragma unroll
    for (int m = 8; m < 8 * U; m <<= 1) d += __shfl_xor_sync(0xffffffffu, d, m);
    const int q = tid;  // A units: threads < 128 U
    if (q < ROWS * U && ((q >> 3) % U) == 0) diag_s[(q & 7) + 8 * ((q >> 3) / U)] = d;
    __syncthreads();
  }

  // ---- epilogue
  const int rl = 32 * (warp & 3) + lane, cb = 32 * (warp >> 2);
  if (MODE == 0) {
    double* P = p.part + (size_t)blockIdx.z * p.M * p.N;
    const int r = r0 + rl;
    if (r < p.M) {
#pragma unroll
      for (int e = 0; e < 32; ++e) {
        const int c = c0 + cb + e;
        if (c < p.N) P[(size_t)c * p.M + r] = (same && cb + e == rl) ? diag_s[rl] : acc[e];
      }
    }
  } else if (MODE == 2) {  // tile column cb + e = channel ch, pair c0 + jj -> ch jp + pair
    double* P = p.part + (size_t)blockIdx.z * p.M * p.N;
    const int r = r0 + rl;
    if (r < p.M) {
#pragma unroll
      for (int e = 0; e < 32; ++e) {
        const int ch = (cb + e) / p.jt, j = c0 + (cb + e) - ch * p.jt;
        if (ch < p.nch && j < p.jp) P[(size_t)(ch * p.jp + j) * p.M + r] = acc[e];
      }
    }
  } else {
    const int pt = r0 + rl;
    if (pt < p.M) {
      const double sc = p.alpha * (p.w ? p.w[pt >> 1] : 1.0);
#pragma unroll
      for (int e = 0; e < 32; ++e) {
        const int i = c0 + cb + e;
        if (i < p.N) {
          double v = acc[e];
          if (MODE == 1 && i < p.nin)
            v = fma(p.B[(size_t)i * p.ldb + i], p.A[(size_t)i * p.lda + pt], v);
          double* o = p.out + (size_t)i * p.ldo + pt;
          *o = p.beta == 0.0 ? sc * v : fma(p.beta, *o, sc * v);
        }
      }
    }
  }
}

template <int MODE, int NLD, int NST, int KC>
int launch(cudaStream_t s, dim3 grid, const Args& a) {
  using C = Cfg<MODE, NLD, NST, KC>;
  static_assert(C::BYTES + (int)sizeof(double) * ROWS + 64 <= 227 * 1024, "shared memory");
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

// one operand (S): 32-real chunks, 3 stages; two operands: 16-real chunks, 4 stages
constexpr int KC_ONE = 32, NST_ONE = 3, KC_TWO = 16, NST_TWO = 4;

inline bool al16(const void* q) { return ((uintptr_t)q & 15) == 0; }

}  // namespace pctc

// EES sums of one atom type (MODE 2): C(s, ch jp + j) = sum_p wpt Re(conj psi_s
// conj(dyp_ch) S_j), j < jp pairs; C column-major [nch jp][ldc], alpha = 1.
int ees_tc_sums(cpstep_ctx* c, const double* psi, const float* sv, long long ld_s,
                const double2* dyp, int nch, int jp, double* C, int ldc) {
  using namespace pctc;
  const int S = c->nstates, K = 2 * c->npts;
  if (nch < 1 || nch > 4 || (ld_s & 3) || !al16(sv) || !al16(psi)) return CPSTEP_ERR_ARG;
  const int jt = ROWS / nch;
  const int tm = cdiv(S, ROWS), tn = cdiv(jp, jt);
  const int want = std::max(1, c->tune.pc_split * c->num_sms / (tm * tn));
  const int kslab = cdiv(cdiv(K, want), 128) * 128;
  const int nsplit = cdiv(K, kslab);
  const int N = nch * jp;
  if (int rc = pc_part_reserve(c, (size_t)nsplit * S * N)) return rc;
  Args p{};
  p.A = psi;
  p.lda = K;
  p.w = c->d_wpt;
  p.M = S;
  p.N = N;
  p.K = K;
  p.kslab = kslab;
  p.part = c->d_pc_part;
  p.err = c->d_dev_err;
  p.sv = sv;
  p.ld_s = ld_s;
  p.dyp = dyp;
  p.ld_d = c->npts;
  p.nch = nch;
  p.jt = jt;
  p.jp = jp;
  if (int rc = launch<2, 2, NST_TWO, KC_TWO>(c->stream, dim3(tm, tn, nsplit), p)) return rc;
  return pc_splitk_reduce_launch(c, nsplit, S, N, 1.0, 0.0, C, ldc, 0);
}

// EES psi force of one atom type (MODE 3): fpsi_s(p) += alpha wpt(p) sum_j
// Z(j, s) (conj(dyp_c) S_a)(p), j = c natm_t + a; Z column-major [S][ldz].
int ees_tc_force(cpstep_ctx* c, const float* sv, long long ld_s, const double2* dyp, int nch,
                 int natm_t, const double* Z, int ldz, double alpha, double* fpsi) {
  using namespace pctc;
  const int S = c->nstates, K = 2 * c->npts;
  if (nch < 1 || nch > 4 || (ld_s & 3) || (ldz & 1) || !al16(sv) || !al16(Z)) return CPSTEP_ERR_ARG;
  Args p{};
  p.B = Z;
  p.ldb = ldz;
  p.w = c->d_wpt;
  p.M = K;
  p.N = S;
  p.K = K;
  p.nin = nch * natm_t;
  p.out = fpsi;
  p.ldo = K;
  p.alpha = alpha;
  p.beta = 1.0;
  p.err = c->d_dev_err;
  p.sv = sv;
  p.ld_s = ld_s;
  p.dyp = dyp;
  p.ld_d = c->npts;
  p.nch = nch;
  p.natm_t = natm_t;
  return launch<3, 2, NST_TWO, KC_TWO>(c->stream, dim3(cdiv(K, ROWS), cdiv(S, ROWS)), p);
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

int pc_backmul_tc_launch(cpstep_ctx* c, const double* Mcm, int ldm, const double* in, int ldi,
                         double* out, int ldo, int nout, int nin, int K, double alpha,
                         double beta, const double* w, bool* used) {
  using namespace pctc;
  *used = false;
  if (!pc_tc_usable(c) || (K & 1) || (ldm & 1) || (ldi & 1) || !al16(Mcm) || !al16(in))
    return CPSTEP_OK;
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
  if (int rc = launch<1, 2, NST_TWO, KC_TWO>(c->stream, dim3(cdiv(K, ROWS), cdiv(nout, ROWS)), p))
    return rc;
  *used = true;
  return CPSTEP_OK;
}
