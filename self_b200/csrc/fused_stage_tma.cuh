// Persistent variant of the fused stage kernel.
//
// One CTA per SM, made of C consumer groups of TPE threads (one thread per
// node).  A group works through the CTA's elements g, g + C, g + 2C, ... and
// owns two shared-memory buffers: for every element its thread 0 issues 1-D
// bulk asynchronous copies (cp.async.bulk, the non-tensor TMA path) of the
// element's contiguous blocks -- solution, the engine's packed geometry record
// (dsdx, nHat, nScale, J, sideInfo), its own face traces and the model fields
// -- into a buffer whose mbarrier counts the bytes in, two elements ahead: the
// copies for element jj + 2 go out as soon as element jj has released its
// buffer.  The number of copy requests per element, not their bytes, is what
// costs, so the per-element pieces that live in separate arrays are packed
// into one record at set-up.  The face threads load the neighbours' trace
// values themselves (coalesced plain loads).  With no separate producer warp,
// ten groups of two warps fill the SM's four schedulers with five warps each
// at 96 registers per thread.
//
// Every wait is bounded (StageArgs::waitCycles): on timeout the group records
// an error word, waits (again bounded) for its other copy in flight and
// returns; the host reports SELFGPU_ERR_TIMEOUT.
//
// Requires an even P (all per-element block sizes are then multiples of 16
// bytes) and 16-byte aligned base pointers; the engine falls back to
// k_fused_stage otherwise.
#pragma once

#include "fused_stage.cuh"

namespace selfgpu {

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded wait: true when the phase with this parity has completed.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, long long cycles) {
  if (mbar_try_wait(bar, parity)) return true;
  const long long t0 = clock64();
  while (true) {
    if (mbar_try_wait(bar, parity)) return true;
    if (clock64() - t0 > cycles) return false;
    __nanosleep(64);
  }
}
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ void named_bar(int id, int nthreads) {
  asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(nthreads) : "memory");
}
__device__ __forceinline__ unsigned ld_acquire(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
// Bounded wait until *p >= v (acquire); false when the budget ran out.
__device__ __forceinline__ bool wait_at_least(const unsigned* p, unsigned v, long long cycles) {
  if (ld_acquire(p) >= v) return true;
  const long long t0 = clock64();
  while (true) {
    if (ld_acquire(p) >= v) return true;
    if (clock64() - t0 > cycles) return false;
    __nanosleep(128);
  }
}

// Runtime layout of one element buffer (byte offsets; -1 = piece absent) and
// of the CTA's shared memory.  Built on the host by make_tma_plan().
struct TmaPlan {
  int groups;      // consumer groups per CTA
  int slotBytes;   // bytes of one element buffer
  int oQ, oDsdx, oNhat, oNs, oJ, oSi, oOwn;  // oDsdx..oSi lie in the packed geometry record
  int oX[5];       // model fields: LSW (H, Hb, fC), SW (topoB, grad), CIG (envG, drag, presc x3 -> oX[2..4])
  int oVelOwn;
  int oMats, oFlags, oSlots, oGroups, groupBytes, smemBytes;
};

// Several RK stages in one launch of k_fused_stage_tma<..., true>: stage s
// (0-based) is RK3 stage s % 3 with the trace and velocity caches of parity
// cur0 + s (vcur0 + s), as selfgpu_model2d's stage-by-stage loop would issue
// them.  Every group runs the same tiles in every stage, so each stage's own
// data (solution, own traces and velocity traces) come from the group itself
// and are copied ahead across the stage boundary.  Only the neighbour traces
// need the other CTAs' stage: a group announces the end of its stage on a
// counter (bar) and, in its next stage, its face warp waits for every
// group's announcement before its first neighbour loads (the copies, the
// flux phase and the divergence sums of that tile go ahead meanwhile).  One
// face warp per tile: P = 8 (one element per group) only.  (Per-tile stage
// flags instead of the one counter, so that no stage waits for the whole
// grid, measured 25-45 % slower: a release fence per tile and an acquire
// load per face thread cost more than the waits they save.)
struct TmaSteps {
  int nStages;
  int nGroups;      // groups of the launch (every one has at least 3 tiles)
  double dt;
  double rkA[3], rkG[3];
  void* tr[2];
  void* vel[2];
  int cur0, vcur0;
  unsigned* bar;    // stage-end counter, zero at launch
};

// Smallest stride >= n values of `bytes` bytes whose byte size is 64 mod 128:
// four consecutive sides then occupy alternate halves of the 32 banks.
__host__ __device__ constexpr int side_stride(int n, int bytes) {
  int k = n;
  while ((k * bytes) % 128 != 64) ++k;
  return k;
}

template <int P, class Phys, typename R>
struct TmaTraits {
  static constexpr int PP = P * P, NV = Phys::NV, NT = Phys::NT, NF = Phys::NF;
  static constexpr int TS = trace_side_stride<P, NT, R>();
  // Elements per group (a tile of consecutive elements).  A P = 4 element
  // (16 nodes) would leave half of its warp's lanes idle: two per one-warp
  // group.  A P = 6 element (36 nodes) on a two-warp group leaves 28 lanes
  // idle: four per five-warp group (144 of 160 lanes), measured 1.14x faster
  // for ShallowWater FP64, 1.12x for CompressibleIdealGas2D FP32 and, with
  // three 128-register groups (below), 1.27x for CompressibleIdealGas2D FP64.
  static constexpr int EPG = (P == 4) ? 2 : ((P == 6) ? 4 : 1);
  static constexpr int TPE = (EPG * PP + 31) / 32 * 32;  // threads per group
  static_assert(TPE >= EPG * 4 * P, "the face phase gives each of the 4P face nodes its own thread");
  // 640 threads (five warps per scheduler at 96 registers) for P = 6 (ten
  // one-element or four four-element groups) and P = 8; up to 20 single-warp
  // groups for P <= 4 (24 in FP32, at 80 registers: 2-6 % faster than 20),
  // which synchronise with the warp barrier (15 for the
  // FP64 CompressibleIdealGas2D and reference-rounding kernels, whose
  // registers would not fit 20: 16 measured 0.6 % slower, 15 with the warp
  // barrier 0.8 % faster than with named barriers).  Larger groups use
  // named barriers 1..15 (barrier 0 is the CTA-wide one).
  // ShallowWater and CompressibleIdealGas2D FP64 at P = 6 run three
  // four-element groups at 128 registers instead: at 96 they spill (measured
  // 108.5 against 113.5 us per stage for ShallowWater on 256x256;
  // CompressibleIdealGas2D's tiles leave room for three groups only anyway:
  // 144 us, against 183 us with one-element groups).  LinearShallowWater and
  // the FP32 forms are faster with four groups (five, at 72 registers with a
  // few spilled words, measured 12-16 % slower in FP32).  The FP32 forms at P = 8 run
  // fourteen groups (896 threads at 72 registers, no spills): against ten,
  // 7-16 % faster per stage on 256x256 meshes and 6 % on 128x128; fifteen (64
  // registers) measured 1.5-22 % slower than fourteen.  Twelve
  // groups (80 registers) run the production FP64
  // ShallowWater and LinearShallowWater kernels (80 registers without spills;
  // CompressibleIdealGas2D FP64 would spill and its shared memory holds ten
  // groups, the reference-rounding build would spill).
  static constexpr int kMaxGroups =
      (P <= 4) ? (((NV == 4 && sizeof(R) == 8) || ref_rounding<R>()) ? 15 : (sizeof(R) == 4 ? 24 : 20))
               : (P == 6 ? ((EPG == 4 && (Phys::kLaggedVelocity || NV == 4) && sizeof(R) == 8) ? 3 : 640 / TPE)
                         : ((sizeof(R) == 4) ? 14 : (NV == 3 && !ref_rounding<R>()) ? 12 : 10));
  static constexpr int kThreadsMax = kMaxGroups * TPE;
  // Per-element compute arrays (bulk type), laid out for conflict-free shared
  // accesses.  A 64-bit shared access is served per half-warp: two threads of
  // a half-warp that touch different words of one bank pair (8-byte word
  // index mod 16) cost an extra pass.
  //  * contravariant fluxes [2][NV][P][P]: a half-warp holds rows j and j + 1.
  //  * node fields of the updated solution, read one line per thread by the
  //    trace tasks: field stride FS = 8 (mod 16) and, for P = 8, the column
  //    index XOR-swizzled per (field, row) so that the column lines and the
  //    row lines of two fields fall into distinct bank pairs; other P pad
  //    rows to P + 1.
  //  * boundary-normal flux [4][SS]: sides SS values apart, SS * sizeof(R) =
  //    64 (mod 128).
  // With two elements per group their arrays follow each other (EB values
  // apart), and the divergence sums go to a separate array (NV P^2 per
  // element) instead of replacing the xi flux, since one element's
  // divergence threads may then span two warps.
  static constexpr bool kSwz = (P == 8);
  static constexpr int RS = kSwz ? P : P + 1;
  static constexpr int FS = kSwz ? PP + 8 : P * RS;
  static constexpr int kU = (NF * FS > 2 * NV * PP) ? NF * FS : 2 * NV * PP;  // node fields alias the fluxes
  static constexpr int SS = side_stride(NV * P, (int)sizeof(R));
  static constexpr int EB = kU + 4 * SS;
  static constexpr int kDiv = EPG > 1 ? NV * PP : 0;  // separate divergence sums per element
  static constexpr int groupBytes = (int)(((EPG * (EB + kDiv)) * sizeof(R) + 127) / 128 * 128);
  // Weak-divergence volume sums: one thread per 2x2 block of nodes and pair
  // of variables.  The xi flux rows are stored with their value pairs
  // XOR-swizzled per row pair (P/2 a power of two), so that the paired loads
  // of a quarter-warp fall into distinct banks.
  static constexpr int HB = P / 2, NVP = (NV + 1) / 2, NB = HB * HB * NVP;
  static_assert(EPG > 1 || NB <= 32, "one element's divergence blocks fit one warp");
  static_assert(EPG * NB <= TPE, "every divergence block has its own thread");
  static constexpr bool kSwzF = (HB & (HB - 1)) == 0;
  // position of value m in row j of the xi flux
  __device__ __forceinline__ static int f0pos(int m, int j) {
    if constexpr (kSwzF) return 2 * ((m >> 1) ^ ((j >> 1) & (HB - 1))) + (m & 1);
    else return m;
  }
  // offset of node (i, j) in field f's block of the node-field array
  __device__ __forceinline__ static int nf(int f, int i, int j) {
    if constexpr (kSwz) return P * j + (i ^ (((j >> 1) ^ (4 * (f & 1))) & (P - 1)));
    else return RS * j + i;
  }
};

template <int P, class Phys, typename R, bool kMulti = false>
__global__ void __launch_bounds__(TmaTraits<P, Phys, R>::kThreadsMax, 1)
    k_fused_stage_tma(const StageArgs a, const TmaPlan pl, const TmaSteps ms) {
  using T = TmaTraits<P, Phys, R>;
  constexpr int NV = T::NV, NT = T::NT, NF = T::NF, PP = T::PP, TS = T::TS, TPE = T::TPE, N = P - 1;
  constexpr int FS = T::FS, SS = T::SS, EPG = T::EPG, EB = T::EB;
  constexpr bool kLSW = (NV == 3 && !Phys::kLaggedVelocity);
  constexpr bool kSW = Phys::kLaggedVelocity;
  // Neighbour traces loaded before phase A (measured per configuration: a
  // gain at P = 8 and for ShallowWater FP64 at P = 6; a loss where the
  // registers they hold across phase A make the kernel spill or crowd it --
  // reference-rounding CompressibleIdealGas2D at P = 8, CompressibleIdealGas2D
  // at P = 6, every model at P = 4)
  constexpr bool kNbrEarly =
      (P == 8) ? !(NV == 4 && ref_rounding<R>()) : (P == 6 && kSW && sizeof(R) == 8);
  // divergence sums as FP64 tensor-core products (phase B): production and
  // FP32-bulk forms at P = 8 and 6 (one element per warp) and 4 (two)
  constexpr bool kDmma = ((P == 8 && EPG == 1) || P == 6) && !ref_rounding<R>();
  constexpr bool kDmma4 = (P == 4 && EPG == 2 && TPE == 32) && !ref_rounding<R>();
  // At P = 8 the products' operand loads read, per half-warp, four rows of
  // the xi flux, the eta flux and the transposed dgMatrix at four columns
  // each; rows two apart would share banks, so these three arrays keep the
  // column index XOR 4 in row pairs 2-3 and 6-7 (the per-node stores of
  // phase A stay conflict-free, as a half-warp stores two whole rows).
  constexpr bool kSw8 = (P == 8) && kDmma;
  auto cswz = [](int c, int r) { return kSw8 ? (c ^ (4 * ((r >> 1) & 1))) : c; };
  auto f0at = [&](int m, int j) { return kSw8 ? P * j + cswz(m, j) : P * j + T::f0pos(m, j); };  // F0(m, j)
  auto f1at = [&](int i, int j) { return P * j + cswz(i, j); };                                  // F1(i, j)
  auto dgat = [&](int m, int i) { return P * m + cswz(i, m); };                                  // dgM(m, i)
  extern __shared__ __align__(128) unsigned char smem[];
  const int C = pl.groups;
  uint64_t* full = reinterpret_cast<uint64_t*>(smem);
  double* sdg = reinterpret_cast<double*>(smem + pl.oMats);
  double* sb = sdg + PP;
  double* sqw = sb + 2 * P;
  double* sqwr = sqw + P;  // 1/w (the FP32-bulk and production FP64 forms)
  // bMatrix and 1/w in the bulk type (FP32-bulk form: rounded copies after 1/w)
  R* sbR = sizeof(R) == 8 ? reinterpret_cast<R*>(sb) : reinterpret_cast<R*>(sqwr + P);
  R* sqwrR = sizeof(R) == 8 ? reinterpret_cast<R*>(sqwr) : sbR + 2 * P;
  volatile int* gflag = reinterpret_cast<volatile int*>(smem + pl.oFlags);
  unsigned char* slots = smem + pl.oSlots;

  if (threadIdx.x == 0) {
    for (int k = 0; k < 2 * C; ++k) mbar_init(&full[k], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  // dgMatrix transposed (sdg[i + P m] = dgM(m, i), the column index swizzled
  // where kSw8): a warp's reads of the columns of its nodes' i (or j) are then
  // consecutive
  for (int k = threadIdx.x; k < PP; k += blockDim.x) sdg[dgat(k / P, k % P)] = a.dgM[k / P + P * (k % P)];
  for (int k = threadIdx.x; k < 2 * P; k += blockDim.x) {
    sb[k] = a.bM[k];
    if constexpr (sizeof(R) == 4) sbR[k] = a.bMf[k];
  }
  for (int k = threadIdx.x; k < P; k += blockDim.x) {
    sqw[k] = a.qw[k];
    sqwr[k] = 1.0 / a.qw[k];
    if constexpr (sizeof(R) == 4) sqwrR[k] = (R)(1.0 / a.qw[k]);
  }
  __syncthreads();
  // Launched as a programmatic dependent of the previous kernel on the stream:
  // let the next launch start its own prologue, then wait until the previous
  // kernel has completed and its writes are visible.  Everything above reads
  // only set-up constants; everything below may read what it wrote or write
  // what it read.  (Both are no-ops for an ordinary launch.)
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
  asm volatile("griddepcontrol.wait;" ::: "memory");

  // Work items are tiles of EPG consecutive elements; the CTA takes tiles
  // blockIdx.x, blockIdx.x + gridDim.x, ...
  const long long nTiles = ((long long)a.nEl + EPG - 1) / EPG;
  const long long nMine =
      (long long)blockIdx.x < nTiles ? (nTiles - blockIdx.x + gridDim.x - 1) / gridDim.x : 0;
  static_assert(!kMulti || EPG == 1, "several stages per launch: one face warp per tile");
  const bool rk = kMulti || (a.mode == MODE_RK);
  const int g = threadIdx.x / TPE;
  const int t = threadIdx.x % TPE;
  if (g >= C) return;
  // work items of group g: its tiles g, g + C, ... of the CTA (nMineG per
  // stage), stage after stage
  const long long nMineG = (long long)g < nMine ? (nMine - g + C - 1) / C : 0;
  const long long nItems = kMulti ? nMineG * ms.nStages : nMineG;
  auto cache_of = [&](void* const* pair, int c0, int st, const void* one) -> const void* {
    return kMulti ? (((c0 + st) & 1) ? pair[1] : pair[0]) : one;  // a stage's input cache (no dynamic index)
  };

  // Group g consumes the CTA's tiles g, g + C, g + 2C, ... through its two
  // buffers; its thread 0 issues the copies of local tile jj + 2 into the
  // buffer that tile jj has just released.  Every piece of a tile is
  // contiguous in global memory (element-major arrays), so a tile is still
  // one bulk copy per piece.
  // the geometry record's kind: FP32 metrics and an FP64 1/J in the FP32-bulk
  // form; FP64 metrics with J (reference roundings), 1/J (production FP64 at
  // P < 8) or no J slot (production FP64 at P = 8, which forms 1/J from dsdx:
  // measured faster there, slower at P = 6)
  constexpr int kGeo = geo_kind<P, R>();
  constexpr GeoRec kRec = geo_rec(P, kGeo);
  const uint32_t qb = NV * PP * 8, gb = kRec.bytes, ob = 4 * TS * sizeof(R);
  const uint32_t vb = kSW ? 8 * P * sizeof(R) : 0;
  uint32_t xb[5] = {0, 0, 0, 0, 0};  // per element
  if constexpr (kLSW) {
    xb[0] = PP * 8;
    xb[1] = 4 * P * 8;
    xb[2] = a.fld[2] ? PP * 8 : 0;
  } else if constexpr (kSW) {
    xb[0] = a.fld[0] ? 4 * P * 8 : 0;
    xb[1] = a.fld[1] ? 2 * PP * 8 : 0;
  } else {
    xb[0] = a.fld[0] ? 2 * PP * 8 : 0;
    xb[1] = a.fld[1] ? PP * 8 : 0;
    xb[2] = xb[3] = xb[4] = a.fld[2] ? 16 * P * 8 : 0;
  }
  auto tile_live = [&](long long k) -> int {  // live elements of the CTA's local tile k
    const long long e0 = (blockIdx.x + k * gridDim.x) * EPG;
    const long long r = (long long)a.nEl - e0;
    return r < EPG ? (int)r : EPG;
  };
  // item w = tile jj of stage st (thread 0 only)
  auto issue = [&](long long w, int st, long long jj) {
    if (w >= nItems) return;
    const long long k = g + jj * C;
    const int buf = (int)(w & 1);
    const long long e = (blockIdx.x + k * gridDim.x) * EPG;  // first element of the tile
    const uint32_t nl = (EPG == 1) ? 1u : (uint32_t)tile_live(k);
    unsigned char* sl = slots + (size_t)(2 * g + buf) * pl.slotBytes;
    uint64_t* bar = &full[2 * g + buf];
    const uint32_t bytes = nl * (qb + gb + ob + vb + xb[0] + xb[1] + xb[2] + xb[3] + xb[4]);
    mbar_arrive_expect_tx(bar, bytes);
    if (a.debugStarve == 1 && blockIdx.x == 0 && k == 0) return;
    const R* trIn = reinterpret_cast<const R*>(cache_of(ms.tr, ms.cur0, st, a.trIn));
    bulk_g2s(sl + pl.oQ, a.q + (size_t)e * NV * PP, nl * qb, bar);
    bulk_g2s(sl + pl.oDsdx, reinterpret_cast<const unsigned char*>(a.geo) + (size_t)e * gb, nl * gb, bar);
    bulk_g2s(sl + pl.oOwn, trIn + (size_t)4 * TS * e, nl * ob, bar);
    if constexpr (kSW)
      bulk_g2s(sl + pl.oVelOwn,
               reinterpret_cast<const R*>(cache_of(ms.vel, ms.vcur0, st, a.velIn)) + (size_t)e * 8 * P, nl * vb,
               bar);
    if constexpr (kLSW) {
      bulk_g2s(sl + pl.oX[0], a.fld[0] + (size_t)e * PP, nl * xb[0], bar);
      bulk_g2s(sl + pl.oX[1], a.fld[1] + (size_t)e * 4 * P, nl * xb[1], bar);
      if (xb[2]) bulk_g2s(sl + pl.oX[2], a.fld[2] + (size_t)e * PP, nl * xb[2], bar);
    } else if constexpr (kSW) {
      if (xb[0]) bulk_g2s(sl + pl.oX[0], a.fld[0] + (size_t)e * 4 * P, nl * xb[0], bar);
      if (xb[1]) bulk_g2s(sl + pl.oX[1], a.fld[1] + (size_t)e * 2 * PP, nl * xb[1], bar);
    } else {
      // environmentalsGradient (2,P,P,2,nEl): variable 1, both components, of each element
      if (xb[0])
        for (uint32_t x = 0; x < nl; ++x)
          bulk_g2s(sl + pl.oX[0] + x * xb[0], a.fld[0] + (size_t)(e + x) * 4 * PP, xb[0], bar);
      // environmentals (P,P,2,nEl): variable 2 (drag) of each element
      if (xb[1])
        for (uint32_t x = 0; x < nl; ++x)
          bulk_g2s(sl + pl.oX[1] + x * xb[1], a.fld[1] + (size_t)(e + x) * 2 * PP + PP, xb[1], bar);
      if (xb[2])
        for (int x = 2; x < 5; ++x) bulk_g2s(sl + pl.oX[x], a.fld[x] + (size_t)e * 16 * P, nl * xb[x], bar);
    }
  };
  if (t == 0) {
    issue(0, 0, 0);  // (a group has at least three tiles per stage when there are several stages)
    issue(1, 0, 1);
  }

  const int barId = 1 + g;
  // a one-warp group synchronises with the warp barrier (no named-barrier
  // limit on the number of groups); larger groups use named barrier 1 + g
  auto group_bar = [&]() {
    if constexpr (TPE == 32) __syncwarp();
    else named_bar(barId, TPE);
  };
  // node phases: thread t serves node n of element ee of the tile
  const int ee = t / PP;
  const int n = t - ee * PP;
  const int i = n % P, j = n / P;
  // Which warp of a one-element group runs the face phase (the other one sums
  // the divergence meanwhile): alternated in pairs of groups so that both
  // kinds of work spread over the SM's four schedulers (warp w runs on w mod
  // 4).  Two-element groups give the divergence blocks to their first
  // threads and the face nodes to their last ones.
  const int faceWarp = (EPG == 1 && TPE >= 64) ? ((g >> 1) & 1) : 0;
  R* gBase = reinterpret_cast<R*>(smem + pl.oGroups + (size_t)g * pl.groupBytes);
  R* gU = gBase + ee * EB;      // this thread's element: fluxes, later node fields
  R* gF1 = gU + NV * PP;        // eta flux [NV][P][P]
  R* gfb = gU + T::kU;          // [4][SS]: [NV][P] per side
  R* gD = (EPG > 1) ? gBase + EPG * EB + ee * NV * PP : gU;  // divergence sums
  constexpr int rNhat = kRec.oNhat, rNs = kRec.oNs, rJ = kRec.oJ, rSi = kRec.oSi;

  int st = 0;        // stage of item w
  long long jj = -1;  // index of item w's tile among the group's tiles
  for (long long w = 0; w < nItems; ++w) {
    if constexpr (kMulti) {
      if (++jj == nMineG) {
        jj = 0;
        ++st;
      }
    } else {
      jj = w;
    }
    const long long k = g + jj * C;
    // this stage's caches and RK coefficients
    const R* trIn = reinterpret_cast<const R*>(cache_of(ms.tr, ms.cur0, st, a.trIn));
    R* trOut = reinterpret_cast<R*>(const_cast<void*>(cache_of(ms.tr, ms.cur0, st + 1, a.trOut)));
    const R* velIn = reinterpret_cast<const R*>(cache_of(ms.vel, ms.vcur0, st, a.velIn));
    R* velOut = reinterpret_cast<R*>(const_cast<void*>(cache_of(ms.vel, ms.vcur0, st + 1, a.velOut)));
    const int m3 = st % 3;
    const double rkA = kMulti ? (m3 == 0 ? ms.rkA[0] : (m3 == 1 ? ms.rkA[1] : ms.rkA[2])) : a.rk_a;
    const double rkG = kMulti ? (m3 == 0 ? ms.rkG[0] : (m3 == 1 ? ms.rkG[1] : ms.rkG[2])) : a.rk_g;
    const double rkGdt = kMulti ? rkG * ms.dt : a.rk_gdt;
    // the stage's first tile reads other CTAs' traces of the previous stage
    const bool gridWait = kMulti && st > 0 && jj == 0;
    const long long e0 = (blockIdx.x + k * gridDim.x) * EPG;
    const int nLive = (EPG == 1) ? 1 : tile_live(k);
    const long long e = e0 + ee;
    const bool active = (t < EPG * PP) && (ee < nLive);
    const int buf = (int)(w & 1);
    const uint32_t par = (uint32_t)((w >> 1) & 1);
    const unsigned char* sl = slots + (size_t)(2 * g + buf) * pl.slotBytes;
    if (t == 0) gflag[g] = mbar_wait(&full[2 * g + buf], par, a.waitCycles) ? 1 : 0;
    group_bar();
    if (!gflag[g]) {
      if (t == 0) {
        if (a.err) atomicExch(a.err, 1);
        // Wait (bounded) once more for this buffer's copies and for those of
        // the group's other buffer, so that none is pending when the CTA exits.
        mbar_wait(&full[2 * g + buf], par, a.waitCycles);
        if (w + 1 < nItems) mbar_wait(&full[2 * g + (buf ^ 1)], (uint32_t)(((w + 1) >> 1) & 1), a.waitCycles);
      }
      break;
    }
    const unsigned char* rec = sl + pl.oDsdx + (size_t)ee * gb;  // this thread's element's geometry record
    const double* sq = reinterpret_cast<const double*>(sl + pl.oQ + (size_t)ee * qb);
    // node auxiliaries of this element, read from the buffer where they are used
    auto node_aux = [&](double na[3]) {
      na[0] = na[1] = na[2] = 0.0;
      if constexpr (kLSW) {
        na[0] = reinterpret_cast<const double*>(sl + pl.oX[0] + ee * xb[0])[n];
        if (pl.oX[2] >= 0) na[1] = reinterpret_cast<const double*>(sl + pl.oX[2] + ee * xb[2])[n];
      } else if constexpr (kSW) {
        if (pl.oX[1] >= 0) {
          const double* gg = reinterpret_cast<const double*>(sl + pl.oX[1] + ee * xb[1]);
          na[0] = gg[2 * n];
          na[1] = gg[2 * n + 1];
        }
      } else {
        if (pl.oX[0] >= 0) {
          const double* gg = reinterpret_cast<const double*>(sl + pl.oX[0] + ee * xb[0]);
          na[0] = gg[2 * n];
          na[1] = gg[2 * n + 1];
        }
        if (pl.oX[1] >= 0) na[2] = reinterpret_cast<const double*>(sl + pl.oX[1] + ee * xb[1])[n];
      }
    };

    // Face threads of this tile (phase C): each serves one face node of one
    // element.  Their neighbour traces (and, ShallowWater, the neighbour's
    // lagged velocity traces) are plain global loads; where kNbrEarly they
    // are issued here, before phase A, so that their latency overlaps the
    // flux computation, otherwise at the start of phase C.
    const int c0 = TPE - EPG * 4 * P;  // first face thread of a multi-element group
    const int cf = (EPG == 1) ? (t & 31) : t - c0;
    const int eC = cf / (4 * P);
    const bool faceOn = ((EPG == 1) ? ((t >> 5) == faceWarp && (t & 31) < 4 * P) : (t >= c0)) && eC < nLive;
    const int cc = cf - eC * 4 * P;
    const int s1 = cc / P, ii = cc % P;
    const unsigned char* recC = sl + pl.oDsdx + (size_t)eC * gb;
    const int* ssi = reinterpret_cast<const int*>(recC + rSi) + 5 * s1;
    R X[NT], velR[2] = {(R)0, (R)0};
    auto load_neighbour = [&]() {
      const long long nb =
          (ssi[4] == 0) ? (long long)TS * (ssi[3] / 10 - 1 + 4 * (long long)(ssi[2] - 1)) : -1;
      const int i2 = (ssi[3] % 10) ? N - ii : ii;
      // (several stages in one launch: through L2, as the SM's L1 may still
      // hold these lines from two stages back)
      auto ld = [](const R* x) -> R { return kMulti ? __ldcg(x) : *x; };
      const R* nbr = trIn + (nb < 0 ? 0 : nb);
#pragma unroll
      for (int kf = 0; kf < NT; ++kf) X[kf] = (nb >= 0) ? ld(nbr + i2 + P * kf) : (R)0;
      if constexpr (kSW)
        if (nb >= 0) {
          const R* vn = velIn + (size_t)2 * P * (ssi[3] / 10 - 1 + 4 * (size_t)(ssi[2] - 1));
          velR[0] = ld(vn + i2);
          velR[1] = ld(vn + i2 + P);
        }
    };
    if constexpr (kNbrEarly)
      if (faceOn && !gridWait) load_neighbour();

    // ---- A: flux auxiliaries, contravariant flux.  The buffer stays valid
    // until the end of phase D, so the solution, J and the node auxiliaries
    // are read again where they are needed instead of living in registers
    // across the face phase.
    R f[NF];
    if (active) {
#pragma unroll
      for (int v = 0; v < NV; ++v) f[v] = (R)sq[n + PP * v];
      Phys::template node_flux<R>(f, a);
      double na[3];
      node_aux(na);
      R Fx[NV], Fy[NV];
      Phys::template flux<R>(f, na, a, Fx, Fy);
      // dsdx planes: (dsdx11, dsdx21) of every node, then (dsdx12, dsdx22)
      R m11, m21, m12, m22;
      if constexpr (kRec.wm == 4) {  // FP32 record: the metric terms already rounded
        const float2* gp = reinterpret_cast<const float2*>(rec);
        const float2 c1 = gp[n], c2 = gp[PP + n];
        m11 = c1.x, m21 = c1.y, m12 = c2.x, m22 = c2.y;
      } else {
        const double2* gp = reinterpret_cast<const double2*>(rec);
        const double2 c1 = gp[n], c2 = gp[PP + n];
        m11 = (R)c1.x, m21 = (R)c1.y, m12 = (R)c2.x, m22 = (R)c2.y;
      }
      R F0[NV], F1[NV];
#pragma unroll
      for (int v = 0; v < NV; ++v) {
        F0[v] = m11 * Fx[v] + m21 * Fy[v];
        F1[v] = m12 * Fx[v] + m22 * Fy[v];
      }
      if constexpr (NV == 4)
        if (a.av) av_volume_add<P, R>(a, n, e, F0, F1);
#pragma unroll
      for (int v = 0; v < NV; ++v) {
        gU[v * PP + f0at(i, j)] = F0[v];
        gF1[v * PP + f1at(i, j)] = F1[v];
      }
    }
    group_bar();  // contravariant fluxes ready

    // ---- B (alongside the face phase C): weak-divergence volume sums, the
    // reference's order per node and variable (VectorDGDivergence_2D,
    // src/SELF_Lagrange.f90):
    //   d = 0;  for m ascending: d = (d + dgM(m,i) F0(m,j)) + dgM(m,j) F1(i,m).
    // A thread sums a 2x2 block of nodes for two variables, so every loaded
    // flux pair and dgMatrix pair serves two nodes.  One-element groups write
    // the sums over the xi flux ([NV][P^2], node-major) once the warp has read
    // it; two-element groups write them to their separate array.
    // Production FP64 and FP32-bulk forms at P = 8 and P = 6: the same sums
    // as FP64 tensor-core products (mma.sync m8n8k4 f64), D(j,i) = sum_m
    // F0(m,j) dgM(m,i) + dgM(m,j) F1(i,m), four chained products per variable
    // over one warp per element (a P = 6 element is padded with zeros to the
    // 8x8 shape; FP32-bulk fluxes are widened exactly to FP64 and the sums
    // rounded back once).  The order of the additions inside a product is the
    // hardware's, so only the forms without the reference's rounding use it.
    // At P = 4 one product covers both elements of a tile: rows and columns
    // 0-3 belong to the first element, 4-7 to the second; the xi product's
    // A rows and the eta product's B columns carry the element's flux, the
    // dgMatrix operand is the same for both, and the two diagonal 4x4 blocks
    // of the sum are the two elements' sums (the off-diagonal ones mix the
    // elements and are dropped).
    if constexpr (kDmma4) {
      const int lane = t & 31, gq = lane >> 2, kq = lane & 3;
      const int eR = gq >> 2, jr = gq & 3;   // the element and node row of this lane's A row / B column
      const R* bU = gBase + eR * EB;
      const R* bF1 = bU + NV * PP;
      const double dg = sdg[dgat(kq, jr)];    // dgM(m = kq, jr): B of the xi product, A of the eta product
      // this lane's sums: row gq, columns 2 kq, 2 kq + 1 -> element kq >> 1
      const bool diag = (eR == (kq >> 1)) && eR < nLive;
      R* bD = gBase + EPG * EB + eR * NV * PP;
      using R2 = typename std::conditional<sizeof(R) == 8, double2, float2>::type;
#pragma unroll
      for (int v = 0; v < NV; ++v) {
        double c0 = 0.0, c1 = 0.0;
        const double aF0 = (double)bU[v * PP + f0at(kq, jr)];  // F0 at (m = kq, j = jr)
        const double bF = (double)bF1[v * PP + f1at(jr, kq)];   // F1 at (i = jr, m = kq)
        asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
                     : "+d"(c0), "+d"(c1)
                     : "d"(aF0), "d"(dg));
        asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
                     : "+d"(c0), "+d"(c1)
                     : "d"(dg), "d"(bF));
        if (diag) {  // D(j = jr, i = 2 (kq & 1)), D(jr, 2 (kq & 1) + 1)
          R2 x;
          x.x = (R)c0;
          x.y = (R)c1;
          reinterpret_cast<R2*>(bD + v * PP + P * jr)[kq & 1] = x;
        }
      }
    } else if constexpr (kDmma) {
      // the warps a tile's face threads leave free take its elements in turn
      // (a one-element group: the warp that is not the face warp)
      constexpr int kDW = (EPG == 1) ? 1 : ((TPE - EPG * 4 * P) / 32 > 0 ? (TPE - EPG * 4 * P) / 32 : 1);
      const int w = t >> 5;
      const bool run = (EPG == 1) ? (w != faceWarp) : (w < kDW);
      for (int eB = (EPG == 1) ? 0 : w; run && eB < nLive; eB += kDW) {  // uniform over the warp
        const R* bU = gBase + eB * EB;
        const R* bF1 = bU + NV * PP;
        R* bD = (EPG > 1) ? gBase + EPG * EB + eB * NV * PP : gBase;
        const int lane = t & 31, gq = lane >> 2, kq = lane & 3;
        double dv[NV][2];
#pragma unroll
        for (int v = 0; v < NV; ++v) {
          double c0 = 0.0, c1 = 0.0;
#pragma unroll
          for (int kk = 0; kk < 2; ++kk) {
            const int m = 4 * kk + kq;
            const bool in = (P == 8) || (gq < P && m < P);  // the zero padding of P = 6
            const double aF0 = in ? (double)bU[v * PP + f0at(m, gq)] : 0.0;  // F0 at (m, j = gq)
            const double dg = in ? sdg[dgat(m, gq)] : 0.0;                    // dgM(m, gq)
            const double bF = in ? (double)bF1[v * PP + f1at(gq, m)] : 0.0;   // F1 at (i = gq, m)
            asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
                         : "+d"(c0), "+d"(c1)
                         : "d"(aF0), "d"(dg));
            asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
                         : "+d"(c0), "+d"(c1)
                         : "d"(dg), "d"(bF));
          }
          dv[v][0] = c0;  // D(j = gq, i = 2 kq), D(gq, 2 kq + 1)
          dv[v][1] = c1;
        }
        if constexpr (EPG == 1) __syncwarp();  // the warp has read the xi flux it overwrites
        using R2 = typename std::conditional<sizeof(R) == 8, double2, float2>::type;
        if (gq < P && 2 * kq + 1 < P) {
#pragma unroll
          for (int v = 0; v < NV; ++v) {
            R2 x;
            x.x = (R)dv[v][0];
            x.y = (R)dv[v][1];
            reinterpret_cast<R2*>(bD + v * PP + P * gq)[kq] = x;
          }
        }
      }
    } else {
      const bool mine = (EPG == 1) ? (TPE < 64 || (t >> 5) != faceWarp) : (t < EPG * T::NB);
      if (mine) {
        using R2 = typename std::conditional<sizeof(R) == 8, double2, float2>::type;
        constexpr int HB = T::HB;
        const int eB = (EPG == 1) ? 0 : t / T::NB;
        const int tb = (EPG == 1) ? (t & 31) : t - eB * T::NB;
        const bool on = (EPG == 1) ? (tb < T::NB) : (eB < nLive);
        const R* bU = gBase + eB * EB;
        const R* bF1 = bU + NV * PP;
        R* bD = (EPG > 1) ? gBase + EPG * EB + eB * NV * PP : gBase;
        const int vp = tb / (HB * HB), rem = tb - vp * (HB * HB), bj = rem / HB, bi = rem - bj * HB;
        const int v0 = 2 * vp;
        const bool two = v0 + 1 < NV;
        R acc[2][2][2];  // [variable of the pair][row offset r (j)][column offset c (i)]
#pragma unroll
        for (int vv = 0; vv < 2; ++vv)
#pragma unroll
          for (int r = 0; r < 2; ++r) acc[vv][r][0] = acc[vv][r][1] = (R)0;
        if (on) {
          const double2* sdg2 = reinterpret_cast<const double2*>(sdg);
#pragma unroll
          for (int mp = 0; mp < HB; ++mp) {
            R f0[2][2][2];  // [vv][r][k]: F0(2 mp + k, 2 bj + r)
            R f1[2][2][2];  // [vv][k][c]: F1(2 bi + c, 2 mp + k)
#pragma unroll
            for (int vv = 0; vv < 2; ++vv) {
              const int v = (vv == 0 || two) ? v0 + vv : v0;
#pragma unroll
              for (int r = 0; r < 2; ++r) {
                const int row = 2 * bj + r;
                const R2 x = reinterpret_cast<const R2*>(bU + v * PP + P * row)[T::f0pos(2 * mp, row) >> 1];
                f0[vv][r][0] = x.x;
                f0[vv][r][1] = x.y;
              }
#pragma unroll
              for (int kq = 0; kq < 2; ++kq) {
                const R2 x = reinterpret_cast<const R2*>(bF1 + v * PP + P * (2 * mp + kq))[bi];
                f1[vv][kq][0] = x.x;
                f1[vv][kq][1] = x.y;
              }
            }
#pragma unroll
            for (int kq = 0; kq < 2; ++kq) {
              const int m = 2 * mp + kq;
              const double2 dI = sdg2[bi + HB * m], dJ = sdg2[bj + HB * m];
              const R gi[2] = {(R)dI.x, (R)dI.y}, gj[2] = {(R)dJ.x, (R)dJ.y};
#pragma unroll
              for (int vv = 0; vv < 2; ++vv)
#pragma unroll
                for (int r = 0; r < 2; ++r)
#pragma unroll
                  for (int c = 0; c < 2; ++c)
                    acc[vv][r][c] = acc[vv][r][c] + gi[c] * f0[vv][r][kq] + gj[r] * f1[vv][kq][c];
            }
          }
        }
        if constexpr (EPG == 1) __syncwarp();  // the warp has read the xi flux it overwrites
        if (on) {
#pragma unroll
          for (int vv = 0; vv < 2; ++vv)
            if (vv == 0 || two)
#pragma unroll
              for (int r = 0; r < 2; ++r) {
                R2 x;
                x.x = acc[vv][r][0];
                x.y = acc[vv][r][1];
                reinterpret_cast<R2*>(bD + (v0 + vv) * PP + P * (2 * bj + r))[bi] = x;
              }
        }
      }
    }

    // ---- C: faces; own traces of this stage's solution come from the cache,
    // the neighbour's were loaded before phase A
    {
      if (faceOn) {
        if (gridWait) {
          // every group has ended the previous stage (its traces are final):
          // the face warp waits alone, the divergence warp goes on meanwhile
          if ((t & 31) == 0 && !wait_at_least(ms.bar, (unsigned)st * (unsigned)ms.nGroups, a.waitCycles))
            gflag[g] = 0;  // checked after phase C
          __syncwarp();
        }
        if (!kNbrEarly || gridWait) load_neighbour();
        const long long eF = e0 + eC;
        const int bcid = ssi[4];
        const bool physical = (bcid != 0) && (ssi[2] == 0);
        const R* own = reinterpret_cast<const R*>(sl + pl.oOwn + (size_t)eC * ob) + s1 * TS;
        R L[NT];
#pragma unroll
        for (int kf = 0; kf < NT; ++kf) L[kf] = own[ii + P * kf];
        double2 nh;  // the face functions round the normal to R first: FP32 records hold it rounded
        double ns;
        if constexpr (kRec.wm == 4) {
          const float2 nf = reinterpret_cast<const float2*>(recC + rNhat)[ii + P * s1];
          nh = make_double2(nf.x, nf.y);
          ns = reinterpret_cast<const float*>(recC + rNs)[ii + P * s1];
        } else {
          nh = reinterpret_cast<const double2*>(recC + rNhat)[ii + P * s1];
          ns = reinterpret_cast<const double*>(recC + rNs)[ii + P * s1];
        }
        double fx[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
        if constexpr (kLSW) {
          fx[0] = reinterpret_cast<const double*>(sl + pl.oX[1] + eC * xb[1])[ii + P * s1];
        } else if constexpr (kSW) {
          if (physical && pl.oX[0] >= 0)
            fx[0] = reinterpret_cast<const double*>(sl + pl.oX[0] + eC * xb[0])[ii + P * s1];
        } else {
          if (physical && pl.oX[2] >= 0) {
            const double* ps = reinterpret_cast<const double*>(sl + pl.oX[2] + eC * xb[2]);
            const double* pp = reinterpret_cast<const double*>(sl + pl.oX[3] + eC * xb[3]);
            const double* pd = reinterpret_cast<const double*>(sl + pl.oX[4] + eC * xb[4]);
            const int b = ii + P * 4 * s1;
            for (int v = 0; v < 4; ++v) fx[v] = ps[b + v * P];
            fx[4] = pp[b];
            fx[5] = pp[b + P];
            fx[6] = pp[b + 3 * P];
            fx[7] = pd[b + P];
            fx[8] = pd[b + 2 * P];
          }
        }
        R velL[2] = {(R)0, (R)0};
        if constexpr (kSW) {
          const R* vo = reinterpret_cast<const R*>(sl + pl.oVelOwn + (size_t)eC * vb);
          velL[0] = vo[ii + P * (0 + 2 * s1)];
          velL[1] = vo[ii + P * (1 + 2 * s1)];
          R* vOut = velOut;
          if constexpr (ref_rounding<R>()) {
            vOut[ii + P * (0 + 2 * (s1 + 4 * eF))] = L[0] / L[2];
            vOut[ii + P * (1 + 2 * (s1 + 4 * eF))] = L[1] / L[2];
          } else {
            const R rH = (R)1 / L[2];
            vOut[ii + P * (0 + 2 * (s1 + 4 * eF))] = L[0] * rH;
            vOut[ii + P * (1 + 2 * (s1 + 4 * eF))] = L[1] * rH;
          }
        }
        R out[NV];
        Phys::template face<R>(bcid, physical, L, X, velL, velR, nh.x, nh.y, ns, fx, a, out);
        if constexpr (NV == 4)
          if (a.av) av_face_add<P, R>(a, s1, ii, eF, ssi, nh.x, nh.y, ns, out);
        R* fb = gBase + eC * EB + T::kU;
#pragma unroll
        for (int v = 0; v < NV; ++v) fb[s1 * SS + v * P + ii] = out[v];
      }
    }
    group_bar();  // flux and face values ready
    if (gridWait && !gflag[g]) {  // the stage-end wait ran out
      if (t == 0) {
        if (a.err) atomicExch(a.err, 1);
        if (w + 1 < nItems) mbar_wait(&full[2 * g + (buf ^ 1)], (uint32_t)(((w + 1) >> 1) & 1), a.waitCycles);
      }
      break;
    }

    // ---- D: weak divergence + lift, 1/J, source, RK update
    double dsdt[NV], qv[NV], Gv[NV];
    if (active) {
      if (rk) {  // RK register from global memory; the lift below hides the latency
#pragma unroll
        for (int v = 0; v < NV; ++v) {
          const size_t gi = n + (size_t)PP * (v + NV * (size_t)e);
          Gv[v] = sizeof(R) == 4 ? (double)a.Gf[gi] : a.G[gi];  // FP32-bulk form: an FP32 register
        }
      }
#pragma unroll
      for (int v = 0; v < NV; ++v) qv[v] = sq[n + PP * v];
      // J of the node (reference-rounding build) or 1/J (the other forms:
      // from the record, or for production FP64 at P = 8 the reciprocal of
      // det(dsdx) = J)
      double Jij;
      if constexpr (kGeo != GEO_NOJ) {
        Jij = reinterpret_cast<const double*>(rec + rJ)[n];
      } else {
        const double2* gp = reinterpret_cast<const double2*>(rec);
        const double2 c1 = gp[n], c2 = gp[PP + n];
        Jij = 1.0 / (c1.x * c2.y - c2.x * c1.y);
      }
      // sources in FP64 in every form (well-balanced topography / gravity terms)
      double Src[NV], na[3];
      node_aux(na);
      Phys::template source<double>(qv, na, a, Src);
      R d[NV];  // volume sums from phase B
#pragma unroll
      for (int v = 0; v < NV; ++v) d[v] = gD[v * PP + n];
      if constexpr (ref_rounding<R>()) {
        // the reference's divisions, rounded as it rounds them (bit-exact form)
        const R wi = (R)sqw[i], wj = (R)sqw[j];
#pragma unroll
        for (int v = 0; v < NV; ++v) {
          const R dv = d[v] + ((R)sb[i + P] * gfb[1 * SS + v * P + j] + (R)sb[i] * gfb[3 * SS + v * P + j]) / wi +
                       ((R)sb[j + P] * gfb[2 * SS + v * P + i] + (R)sb[j] * gfb[0 * SS + v * P + i]) / wj;
          dsdt[v] = Src[v] - (double)dv / Jij;
        }
      } else {
        // FP32 bulk and production FP64: products with the reciprocals of the
        // weights, and by 1/J
        const R rwi = sqwrR[i], rwj = sqwrR[j];
        const R bi0 = sbR[i], bi1 = sbR[i + P], bj0 = sbR[j], bj1 = sbR[j + P];
        const double rJ = Jij;
#pragma unroll
        for (int v = 0; v < NV; ++v) {
          const R dv = d[v] + (bi1 * gfb[1 * SS + v * P + j] + bi0 * gfb[3 * SS + v * P + j]) * rwi +
                       (bj1 * gfb[2 * SS + v * P + i] + bj0 * gfb[0 * SS + v * P + i]) * rwj;
          dsdt[v] = Src[v] - (double)dv * rJ;
        }
      }
    }
    group_bar();  // every thread is done reading the flux arrays and the buffer
    if (t == 0) {  // refill the buffer: generic-proxy reads before the async-proxy writes
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      if (!kMulti || jj + 2 < nMineG) issue(w + 2, st, jj + 2);
      else issue(w + 2, st + 1, jj + 2 - nMineG);
    }
    if (!rk) {
      if (active)
#pragma unroll
        for (int v = 0; v < NV; ++v) a.dSdt[n + (size_t)PP * (v + NV * (size_t)e)] = dsdt[v];
      continue;
    }
    if (active) {
      const double gdt = a.dtElem ? rkG * a.dtElem[e] : rkGdt;
#pragma unroll
      for (int v = 0; v < NV; ++v) {
        const size_t gi = n + (size_t)PP * (v + NV * (size_t)e);
        const double Gn = rkA * Gv[v] + dsdt[v];
        if constexpr (sizeof(R) == 4) a.Gf[gi] = (float)Gn;  // the solution update uses the FP64 value
        else a.G[gi] = Gn;
        const double qn = qv[v] + gdt * Gn;
        a.q[gi] = qn;
        f[v] = (R)qn;
      }
      Phys::template node<R>(f, a);
#pragma unroll
      for (int v = 0; v < NF; ++v) gU[v * FS + T::nf(v, i, j)] = f[v];
    }
    group_bar();

    // ---- E: traces of the updated solution -> trace cache.  One task per
    // (element, field, line, orientation) reads the line's P values once and
    // forms both of its end traces (BoundaryInterp, src/SELF_Lagrange.f90:
    // 2241-2270): column l gives S (side 0) and N (side 2), row l gives W (3)
    // and E (1).  Tasks are numbered by field pair, orientation, field, line,
    // so that for P = 8 a half-warp reads the column lines (or the row lines)
    // of two fields.
    {
      // P = 8 numbers the tasks by field pair (an odd NT leaves the last
      // pair's second half idle); the padded layouts of the other P number
      // them by orientation, field, line, with no idle tasks
      constexpr int NTp = T::kSwz ? (NT + 1) / 2 * 2 : NT;
      constexpr int TPEl = 2 * NTp * P;  // tasks per element
      // a one-element group's face warp starts one warp later, so the other
      // warp takes the last, partial round
      const int k0 = (EPG == 1) ? (faceWarp ? t : (t + 32) % TPE) : t;
      for (int kk = k0; kk < EPG * TPEl; kk += TPE) {
        const int eE = kk / TPEl, ks = kk - eE * TPEl;
        if (eE >= nLive) continue;
        int row, fi, l;
        if constexpr (T::kSwz) {
          const int fp = ks / (4 * P), r = ks - fp * 4 * P, r2 = r - (r / (2 * P)) * 2 * P, fs = r2 / P;
          row = r / (2 * P);
          l = r2 - fs * P;
          fi = 2 * fp + fs;
          if (fi >= NT) continue;
        } else {
          row = ks / (NT * P);
          const int r = ks - row * NT * P;
          fi = r / P;
          l = r - fi * P;
        }
        const R* fv = gBase + eE * EB + fi * FS;
        R lo = (R)0, hi = (R)0;
#pragma unroll
        for (int m = 0; m < P; ++m) {
          const R x = fv[row ? T::nf(fi, m, l) : T::nf(fi, l, m)];
          lo = lo + bm_left<R>(a, m) * x;  // kernel-parameter constants (m is unrolled)
          hi = hi + bm_right<R, P>(a, m) * x;
        }
        R* o = trOut + (size_t)4 * TS * (e0 + eE);
        o[l + P * fi + TS * (row ? 3 : 0)] = lo;
        o[l + P * fi + TS * (row ? 1 : 2)] = hi;
      }
    }
    // no barrier here: the next tile's post-wait barrier orders the reuse of the arrays
    if constexpr (kMulti) {
      // This tile's solution, traces and velocity traces are read again by
      // bulk copies (async proxy) in the next stage: the copies of tiles 0
      // and 1 go out during this stage's last two tiles, the others during
      // the next stage, so a proxy fence after tiles 0, 1 and the last one
      // orders every write before the copy that reads it.
      if (jj <= 1 || jj == nMineG - 1) asm volatile("fence.proxy.async.global;" ::: "memory");
      if (jj == nMineG - 1 && st + 1 < ms.nStages) {  // the group's stage ends: announce it
        group_bar();
        if (t == 0 && !(a.debugStarve == 2 && blockIdx.x == 0 && g == 0)) {
          __threadfence();
          atomicAdd(ms.bar, 1u);
        }
      }
    }
  }
}

// Host-side plan for k_fused_stage_tma given the smem budget.
template <int P, class Phys, typename R>
inline bool make_tma_plan(const StageArgs& a, int smemLimit, TmaPlan& pl, int maxGroups = 0) {
  using T = TmaTraits<P, Phys, R>;
  constexpr int PP = T::PP, NV = T::NV, TS = T::TS, EPG = T::EPG;
  constexpr bool kLSW = (NV == 3 && !Phys::kLaggedVelocity);
  constexpr bool kSW = Phys::kLaggedVelocity;
  if (P % 2 != 0) return false;
  int o = 0;
  auto put = [&](int bytes) {  // one piece of a tile: EPG elements' blocks back to back
    int at = o;
    o += (EPG * bytes + 15) / 16 * 16;
    return at;
  };
  if (!a.geo) return false;
  pl.oQ = put(NV * PP * 8);
  constexpr GeoRec gr = geo_rec(P, geo_kind<P, R>());
  pl.oDsdx = put(gr.bytes);  // records: dsdx, nHat, nScale, [J or 1/J,] sideInfo
  pl.oNhat = pl.oDsdx + gr.oNhat;  // (offsets within the first element's record)
  pl.oNs = pl.oDsdx + gr.oNs;
  pl.oJ = pl.oDsdx + gr.oJ;
  pl.oSi = pl.oDsdx + gr.oSi;
  pl.oOwn = put(4 * TS * (int)sizeof(R));
  for (int x = 0; x < 5; ++x) pl.oX[x] = -1;
  pl.oVelOwn = -1;
  if (kLSW) {
    pl.oX[0] = put(PP * 8);
    pl.oX[1] = put(4 * P * 8);
    if (a.fld[2]) pl.oX[2] = put(PP * 8);
  } else if (kSW) {
    if (a.fld[0]) pl.oX[0] = put(4 * P * 8);
    if (a.fld[1]) pl.oX[1] = put(2 * PP * 8);
    pl.oVelOwn = put(8 * P * (int)sizeof(R));
  } else {
    if (a.fld[0]) pl.oX[0] = put(2 * PP * 8);
    if (a.fld[1]) pl.oX[1] = put(PP * 8);
    if (a.fld[2])
      for (int x = 2; x < 5; ++x) pl.oX[x] = put(16 * P * 8);
  }
  pl.slotBytes = (o + 127) / 128 * 128;
  pl.groupBytes = T::groupBytes;
  const int cMax = (maxGroups > 0 && maxGroups < T::kMaxGroups) ? maxGroups : T::kMaxGroups;
  for (int C = cMax; C >= 1; --C) {
    int s = 0;
    s += 2 * C * 8;  // barriers
    s = (s + 15) / 16 * 16;
    const int oMats = s;
    s += (PP + 4 * P) * 8;  // dgMatrix, bMatrix, weights, reciprocal weights
    if (sizeof(R) == 4) s += (3 * P * 4 + 15) / 16 * 16;  // their FP32 copies
    const int oFlags = s;
    s += C * 4;  // group flags
    s = (s + 127) / 128 * 128;
    const int oSlots = s;
    s += 2 * C * pl.slotBytes;
    const int oGroups = s;
    s += C * pl.groupBytes;
    if (s <= smemLimit) {
      pl.groups = C;
      pl.oMats = oMats;
      pl.oFlags = oFlags;
      pl.oSlots = oSlots;
      pl.oGroups = oGroups;
      pl.smemBytes = s;
      return true;
    }
  }
  return false;
}

}  // namespace selfgpu
