// tc_count.cuh -- clean-site counts of every pair on the 5th-generation tensor cores (tcgen05, INT8).
//
// For a pair (i, j) the 4x4 table of clean-site base combinations is N_ab(i, j) = sum_k x_i[k][a] x_j[k][b], where
// x_s[k][c] = 1 when sequence s has the clean base c (A, C, G, T = 0..3) at column k. Stacking the four class
// indicator rows of 32 sequences gives A' (128 rows, K = columns); of 64 sequences, B' (256 rows). One
// tcgen05.mma of kind::i8 (M = 128, N = 256, K = 32, u8 x u8 -> s32 in tensor memory) per 32 columns
// accumulates D = A' B'^T, whose 4x4 blocks are the pairs' tables. The epilogue turns each table into the seven
// clean-site aggregates the pair kernel needs (jointly clean sites, matches, A<->G and C<->T transitions, and the
// A, C, G base counts over both sequences) and stores one record per pair slot of [band rows][band columns]: eight
// uint16 (16 bytes, the eighth unused) when the caller asks for them (agg16: the engine's runs do when 32 L < 65536,
// so that the pair kernel can write the final x16 aggregates, at most 32 L, back into the same slot), else eight
// int32 (32 bytes). The pair kernel reads a record with one vector load.
//
// Operand image in HBM (built by onehot_kernel from the compressed codes): per 128-column stage s and 32-sequence
// block b a 16 KB block at (s * NB + b) * 16 KB, in the canonical K-major layout without swizzle: row r =
// 4 * sequence + class, row group g = r / 8 at g * 1024 B, 16-byte column chunk c at + c * 128 B, row r % 8 at
// + (r % 8) * 16 B. Descriptor: leading (K) byte offset 128, stride (8-row group) byte offset 1024. A B' tile is
// two consecutive blocks of the same stage (32 KB, row groups 16..31 continue at 16 KB).
//
// One CTA per tile of 32 rows x 64 columns, 128 threads: thread 0 issues the bulk copies (cp.async.bulk with
// mbarrier transaction counts) into a 2-stage ring, thread 32 issues the MMAs and commits each stage back to its
// producer barrier, then all four warps read the accumulator (warp w holds TMEM lanes 32w..32w+31). Every wait
// is bounded by a deadline on the global nanosecond timer (TcArgs::wait_ns per wait). When a wait gives up, the
// CTA records an error word, lets its copies in flight land, waits (bounded again) for the MMAs it issued to
// complete, and only then frees its tensor memory; its aggregates are not stored and the run reports the
// error.
#pragma once
#include <stdint.h>

namespace tn93 {

constexpr int kTcRows = 32;                     // sequences per A' tile (128 rows of 4 classes)
constexpr int kTcCols = 64;                     // sequences per B' tile (256 rows)
constexpr int kTcStageK = 128;                  // columns (bytes) per pipeline stage
constexpr int kTcBlockBytes = 32 * 4 * kTcStageK;  // one 32-sequence block of one stage: 16 KB
constexpr int kTcStages = 2;
constexpr int kTcStageBytes = 3 * kTcBlockBytes;   // A (one block) + B (two blocks)
constexpr size_t kTcSmem = (size_t)kTcStages * kTcStageBytes + 1024;
constexpr uint64_t kTcWaitNs = 200ull * 1000 * 1000;  // default limit of one bounded wait: 200 ms

struct TcArgs {
  const uint8_t *onehot;  // operand image
  long NB;                // 32-sequence blocks in the image (the last B' tile reads one block past the data)
  long KS;                // 128-column stages
  long N, n1;             // sequences; first column sequence under -s
  bool cross;
  long r0, r1;            // band rows
  long ncols, colbase;    // output row stride and first column it holds
  long cstart;            // first column tile (a multiple of 64 past 0)
  long cend;              // columns at or past cend are not stored (a chunk of the columns; N for all of them)
  void *agg;              // [r1 - r0][ncols] records of 8 uint16 when agg16 (every aggregate < 65536), else 8 int32
  int agg16;
  unsigned long long *err;  // set when a wait gave up
  uint64_t wait_ns;         // limit of each bounded wait (global timer nanoseconds)
  long skip_fill_block;     // test hook: this block skips its first stage copy (-1: none), so a wait runs out
};

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count)
{
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity)
{
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.b32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

__device__ __forceinline__ uint64_t global_ns()
{
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// bounded wait: false when limit_ns passed on the global timer first (the timer is read every 64 polls; a cap on
// the polls themselves bounds the wait even if the timer were to stall)
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, uint64_t limit_ns)
{
  const uint64_t t0 = global_ns();
  for (uint32_t it = 0; it < (1u << 30); it++) {
    if (mbar_try_wait(bar, parity)) return true;
    if ((it & 63) == 63 && global_ns() - t0 > limit_ns) return false;
  }
  return false;
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes)
{
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}

__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar)
{
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}

// K-major, no swizzle: start address, leading (K) byte offset, stride (8-row group) byte offset, version 1
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo)
{
  return (uint64_t)((saddr >> 4) & 0x3FFF) | ((uint64_t)((lbo >> 4) & 0x3FFF) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFF) << 32) | (1ull << 46);
}

// kind::i8 instruction descriptor: s32 accumulator, u8 x u8, both K-major, N = 256, M = 128
constexpr uint32_t kTcIdesc = (2u << 4) | ((uint32_t)(256 >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);

__device__ __forceinline__ void umma_i8(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t accumulate)
{
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(kTcIdesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}

__device__ __forceinline__ void umma_commit(uint64_t *bar)
{
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&v)[16])
{
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15}, [%16];"
      : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]), "=r"(v[8]),
        "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// one thread per (sequence, 16 columns): the four class rows' 16 bytes of the operand image, for the sequences
// [seq0, seq0 + nseq) (seq0 and nseq multiples of 32; sequences at or past N get zero rows)
__device__ __forceinline__ void onehot_body(const uint8_t *__restrict__ cc, long N, long Lc, long NB, long KS,
                                            uint8_t *img, long seq0, long nseq, long bx)
{
  const long t = bx * 256l + threadIdx.x;
  const long nchunk = KS * (kTcStageK / 16);
  if (t >= nseq * nchunk) return;
  const long seq = seq0 + t / nchunk, ch = t % nchunk;
  const long s = ch / (kTcStageK / 16), c = ch % (kTcStageK / 16);
  const long k0 = ch * 16;
  uint8_t code[16];
#pragma unroll
  for (int q = 0; q < 16; q++) code[q] = (seq < N && k0 + q < Lc) ? cc[seq * Lc + k0 + q] : (uint8_t)17;
  const long b = seq / 32, sl = seq % 32;
  uint8_t *blk = img + ((size_t)s * NB + b) * kTcBlockBytes;
#pragma unroll
  for (int cls = 0; cls < 4; cls++) {
    const int r = (int)sl * 4 + cls;
    uint32_t w[4];
#pragma unroll
    for (int q = 0; q < 4; q++)
      w[q] = (uint32_t)(code[4 * q] == cls) | ((uint32_t)(code[4 * q + 1] == cls) << 8) |
             ((uint32_t)(code[4 * q + 2] == cls) << 16) | ((uint32_t)(code[4 * q + 3] == cls) << 24);
    *reinterpret_cast<uint4 *>(blk + (r / 8) * 1024 + c * 128 + (r % 8) * 16) = make_uint4(w[0], w[1], w[2], w[3]);
  }
}

__global__ void onehot_kernel(const uint8_t *__restrict__ cc, long N, long Lc, long NB, long KS, uint8_t *img,
                              long seq0, long nseq)
{
  onehot_body(cc, N, Lc, NB, KS, img, seq0, nseq, blockIdx.x);
}

// Reads the accumulator of tile (i0, j0) (tensor memory from tacc, lane quarter q = 32 rows: sequences
// i0 + 8q .. i0 + 8q + 7, four class rows each; the 16-column chunks c16_0 .. c16_0 + c16_n - 1, 4 column sequences
// each) and stores each pair's record. All 32 lanes of the warp call it.
__device__ __forceinline__ void tc_tile_epilogue(const TcArgs &a, long i0, long j0, uint32_t tacc, int q, int lane,
                                                 int c16_0 = 0, int c16_n = 256 / 16)
{
  const int il = q * 8 + lane / 4, cls = lane & 3;
  const long i = i0 + il;
  for (int c16 = c16_0; c16 < c16_0 + c16_n; c16++) {
    uint32_t v[16];
    tmem_ld16(tacc + ((uint32_t)(q * 32) << 16) + (uint32_t)(c16 * 16), v);
    // v[4 * jj + b] = N_{cls, b}(i, j = 4 * c16 + jj)
    int T[4], dg[4], ag[4], ct[4], col[4][4], rowm[4];
#pragma unroll
    for (int jj = 0; jj < 4; jj++) {
      const int n0 = (int)v[4 * jj], n1 = (int)v[4 * jj + 1], n2 = (int)v[4 * jj + 2], n3 = (int)v[4 * jj + 3];
      rowm[jj] = n0 + n1 + n2 + n3;
      T[jj] = rowm[jj];
      dg[jj] = cls == 0 ? n0 : cls == 1 ? n1 : cls == 2 ? n2 : n3;
      ag[jj] = cls == 0 ? n2 : cls == 2 ? n0 : 0;
      ct[jj] = cls == 1 ? n3 : cls == 3 ? n1 : 0;
      col[jj][0] = n0;
      col[jj][1] = n1;
      col[jj][2] = n2;
      col[jj][3] = n3;
    }
    // totals over the four class rows of sequence i (lanes 4m..4m+3)
#pragma unroll
    for (int o = 1; o < 4; o <<= 1)
#pragma unroll
      for (int jj = 0; jj < 4; jj++) {
        T[jj] += __shfl_xor_sync(0xffffffffu, T[jj], o);
        dg[jj] += __shfl_xor_sync(0xffffffffu, dg[jj], o);
        ag[jj] += __shfl_xor_sync(0xffffffffu, ag[jj], o);
        ct[jj] += __shfl_xor_sync(0xffffffffu, ct[jj], o);
#pragma unroll
        for (int b = 0; b < 3; b++) col[jj][b] += __shfl_xor_sync(0xffffffffu, col[jj][b], o);
      }
    // this lane finishes column jj = cls: base counts of A, C, G over both sequences
    const int base = lane & ~3;
    int out[7] = {0, 0, 0, 0, 0, 0, 0};
#pragma unroll
    for (int jj = 0; jj < 4; jj++) {
      const int rA = __shfl_sync(0xffffffffu, rowm[jj], base + 0);
      const int rC = __shfl_sync(0xffffffffu, rowm[jj], base + 1);
      const int rG = __shfl_sync(0xffffffffu, rowm[jj], base + 2);
      if (jj == cls) {
        out[0] = T[jj];
        out[1] = dg[jj];
        out[2] = ag[jj];
        out[3] = ct[jj];
        out[4] = rA + col[jj][0];
        out[5] = rC + col[jj][1];
        out[6] = rG + col[jj][2];
      }
    }
    const long j = j0 + 4 * c16 + cls;
    const long lb = a.cross ? a.n1 : i + 1;
    if (i >= a.r0 && i < a.r1 && j >= lb && j >= a.colbase && j < a.N && j < a.cend) {
      const size_t at = (size_t)(i - a.r0) * a.ncols + (j - a.colbase);
      if (a.agg16) {
        reinterpret_cast<uint4 *>(a.agg)[at] =
            make_uint4((uint32_t)out[0] | (uint32_t)out[1] << 16, (uint32_t)out[2] | (uint32_t)out[3] << 16,
                       (uint32_t)out[4] | (uint32_t)out[5] << 16, (uint32_t)out[6]);
      } else {
        uint4 *dst = reinterpret_cast<uint4 *>(a.agg) + 2 * at;
        dst[0] = make_uint4((uint32_t)out[0], (uint32_t)out[1], (uint32_t)out[2], (uint32_t)out[3]);
        dst[1] = make_uint4((uint32_t)out[4], (uint32_t)out[5], (uint32_t)out[6], 0u);
      }
    }
  }
}

// One tile: A' = the 32 sequences from i0 (a multiple of 32), B' = the 64 from j0 (a multiple of 32). All 128
// threads of the block call it with the same arguments.
__device__ __forceinline__ void count_tc_tile(const TcArgs &a, long i0, long j0)
{
  extern __shared__ __align__(1024) unsigned char tsm[];
  __shared__ __align__(8) uint64_t full[kTcStages], empty[kTcStages], done;
  __shared__ uint32_t tmem_base;
  __shared__ int abort_flag;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  // block-uniform exit: no valid pair in the tile
  if (i0 >= a.r1 || j0 >= a.N || j0 >= a.cend) return;
  if (!a.cross && j0 + kTcCols - 1 <= i0) return;
  if (a.cross && j0 + kTcCols <= a.n1) return;
  // 1 KB aligned stage ring
  unsigned char *ring = (unsigned char *)(((uintptr_t)tsm + 1023) & ~(uintptr_t)1023);
  if (threadIdx.x == 0) {
    for (int s = 0; s < kTcStages; s++) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    mbar_init(&done, 1);
    abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base)),
                 "r"(256u));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_base;
  const long KS = a.KS;
  const long ab = (i0 / 32), bb = (j0 / 32);
  int fills[kTcStages] = {0, 0};
  const uint64_t lim = a.wait_ns;
  if (threadIdx.x == 0) {
    // producer: stage ring of A (16 KB) + B (32 KB)
    const bool skip_first = a.skip_fill_block >= 0 &&
                            (long)blockIdx.y * gridDim.x + blockIdx.x == a.skip_fill_block;
    for (long k = 0; k < KS; k++) {
      const int s = (int)(k % kTcStages);
      if (k >= kTcStages && !mbar_wait(&empty[s], (uint32_t)(((k / kTcStages) - 1) & 1), lim)) {
        atomicExch(&abort_flag, 1);
        break;
      }
      if (*(volatile int *)&abort_flag) break;
      if (k == 0 && skip_first) continue;  // test hook: stage 0 never fills, so the MMA issuer's wait runs out
      unsigned char *dst = ring + (size_t)s * kTcStageBytes;
      mbar_arrive_expect_tx(&full[s], (uint32_t)kTcStageBytes);
      bulk_g2s(dst, a.onehot + ((size_t)k * a.NB + ab) * kTcBlockBytes, kTcBlockBytes, &full[s]);
      bulk_g2s(dst + kTcBlockBytes, a.onehot + ((size_t)k * a.NB + bb) * kTcBlockBytes, 2 * kTcBlockBytes, &full[s]);
      fills[s]++;
    }
  } else if (threadIdx.x == 32) {
    // MMA issuer
    long k = 0;
    for (; k < KS; k++) {
      const int s = (int)(k % kTcStages);
      if (!mbar_wait(&full[s], (uint32_t)((k / kTcStages) & 1), lim)) {
        atomicExch(&abort_flag, 1);
        break;
      }
      tc_fence_after();
      const uint32_t sa = smem_u32(ring + (size_t)s * kTcStageBytes), sb = sa + kTcBlockBytes;
#pragma unroll
      for (int kk = 0; kk < kTcStageK / 32; kk++)
        umma_i8(tmem, umma_desc(sa + kk * 256, 128, 1024), umma_desc(sb + kk * 256, 128, 1024),
                (k > 0 || kk > 0) ? 1u : 0u);
      umma_commit(&empty[s]);
    }
    umma_commit(&done);  // arrives when every MMA issued above has completed
  }
  // epilogue: all four warps (reconverged: tcgen05.ld is warp-collective)
  __syncwarp();
  const bool ok = __all_sync(0xffffffffu, mbar_wait(&done, 0, lim));
  tc_fence_after();
  const bool go = __all_sync(0xffffffffu, ok && !*(volatile int *)&abort_flag);
  if (go) tc_tile_epilogue(a, i0, j0, tmem, warp, lane);
  // On a timeout: report it, let the last fill of each stage land before the ring is released (a stage is
  // refilled only after its previous fill was consumed, so only the last fill can still be in flight), and make
  // sure every MMA this CTA issued has completed before its tensor memory is freed: the issuer commits `done`
  // after its last MMA on every path, so a second bounded wait on it drains them when the first one gave up.
  if (!go && threadIdx.x == 0) {
    atomicAdd(a.err, 1ull);
    for (int s = 0; s < kTcStages; s++)
      if (fills[s]) mbar_wait(&full[s], (uint32_t)((fills[s] - 1) & 1), lim);
    if (!ok) mbar_wait(&done, 0, lim);
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(256u));
}

// the tiles of one band: A' tiles start at the band's first row rounded down to a 32-sequence block
__global__ void __launch_bounds__(128) count_tc_kernel(TcArgs a)
{
  count_tc_tile(a, (a.r0 / kTcRows) * kTcRows + blockIdx.y * (long)kTcRows, a.cstart + blockIdx.x * (long)kTcCols);
}

// a batch of alignments: block b is tile tiles[b] = (alignment, first row, first column)
__global__ void __launch_bounds__(128) count_tc_batch_kernel(const TcArgs *descs, const int4 *tiles)
{
  const int4 t = tiles[blockIdx.x];
  count_tc_tile(descs[t.x], t.y, t.z);
}

// ---- persistent form ----------------------------------------------------------------------------------------
// One CTA per SM loops over the tiles (t = blockIdx.x, + gridDim.x, ...), with its roles in separate warps:
//   warp 0 (one lane)  producer: the A' and B' blocks of every stage into a 4-stage ring (cp.async.bulk, mbarrier
//                      transaction counts);
//   warp 1 (one lane)  MMA issuer: 4 tcgen05.mma per stage into one of two accumulators (2 x 256 tensor-memory
//                      columns), each stage committed back to the producer, each finished tile to the epilogue;
//   warps 2-9          epilogue: warp w reads tensor-memory lanes 32 (w % 4) .. +31 of a finished accumulator,
//                      columns 128 ((w - 2) / 4) .. +127, stores the records and hands the accumulator back to the
//                      MMA issuer (eight warps, so that the epilogue keeps up with the MMAs).
// So tile t's epilogue overlaps tile t+1's copies and MMAs. Every wait is bounded (TcArgs::wait_ns); a wait that
// gives up stops every role, and the CTA lets its copies land and its MMAs complete (bounded) before it frees its
// tensor memory. Tiles come from a grid over one band (tiles == nullptr: the count_tc_kernel grid of `ga`) or
// from a list of (descriptor, first row, first column) (a batch of alignments).
constexpr int kPStages = 4;
constexpr size_t kPSmem = (size_t)kPStages * kTcStageBytes + 1024;

__device__ __forceinline__ void mbar_arrive(uint64_t *bar)
{
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ bool tc_tile_valid(const TcArgs &a, long i0, long j0)
{
  if (i0 >= a.r1 || j0 >= a.N || j0 >= a.cend) return false;
  if (!a.cross && j0 + kTcCols - 1 <= i0) return false;
  if (a.cross && j0 + kTcCols <= a.n1) return false;
  return true;
}

constexpr int kPEpiWarps = 8;
constexpr int kPThreads = 32 * (2 + kPEpiWarps);

__global__ void __launch_bounds__(kPThreads, 1)
    count_tc_persist_kernel(TcArgs ga, const TcArgs *descs, const int4 *tiles, int ntiles)
{
  extern __shared__ __align__(1024) unsigned char tsm[];
  __shared__ __align__(8) uint64_t full[kPStages], empty[kPStages], accf[2], acce[2], done;
  __shared__ uint32_t tmem_base;
  __shared__ int abort_flag;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const bool listed = tiles != nullptr;
  const long rt0 = listed ? 0 : ga.r0 / kTcRows * kTcRows;
  const long ntx = listed ? 1 : (ga.N - ga.cstart + kTcCols - 1) / kTcCols;
  const long ntot = listed ? (long)ntiles : ntx * ((ga.r1 - rt0 + kTcRows - 1) / kTcRows);
  const uint64_t lim = ga.wait_ns;
  auto tile = [&](long t, const TcArgs *&A, long &i0, long &j0) -> bool {
    if (listed) {
      const int4 x = tiles[t];
      A = &descs[x.x];
      i0 = x.y;
      j0 = x.z;
    } else {
      A = &ga;
      i0 = rt0 + (t / ntx) * kTcRows;
      j0 = ga.cstart + (t % ntx) * kTcCols;
    }
    return tc_tile_valid(*A, i0, j0);
  };
  unsigned char *ring = (unsigned char *)(((uintptr_t)tsm + 1023) & ~(uintptr_t)1023);
  if (threadIdx.x == 0) {
    for (int s = 0; s < kPStages; s++) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    for (int b = 0; b < 2; b++) {
      mbar_init(&accf[b], 1);
      mbar_init(&acce[b], kPEpiWarps);
    }
    mbar_init(&done, 1);
    abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base)),
                 "r"(512u));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_base;
  // producer state kept for the drain: the phase of each stage's last fill (-1: never filled)
  long last_phase[kPStages] = {-1, -1, -1, -1};
  if (warp == 0 && lane == 0) {
    bool skip = ga.skip_fill_block >= 0 && (long)blockIdx.x == ga.skip_fill_block;
    uint32_t g = 0;
    for (long t = blockIdx.x; t < ntot && !*(volatile int *)&abort_flag; t += gridDim.x) {
      const TcArgs *A;
      long i0, j0;
      if (!tile(t, A, i0, j0)) continue;
      const long ab = i0 / 32, bb = j0 / 32;
      for (long k = 0; k < A->KS; k++, g++) {
        const int s = (int)(g % kPStages);
        if (g >= kPStages && !mbar_wait(&empty[s], ((g / kPStages) - 1) & 1, lim)) {
          atomicExch(&abort_flag, 1);
          break;
        }
        if (*(volatile int *)&abort_flag) break;
        if (skip) {  // test hook: this stage never fills, so the MMA issuer's wait runs out
          skip = false;
          continue;
        }
        unsigned char *dst = ring + (size_t)s * kTcStageBytes;
        mbar_arrive_expect_tx(&full[s], (uint32_t)kTcStageBytes);
        bulk_g2s(dst, A->onehot + ((size_t)k * A->NB + ab) * kTcBlockBytes, kTcBlockBytes, &full[s]);
        bulk_g2s(dst + kTcBlockBytes, A->onehot + ((size_t)k * A->NB + bb) * kTcBlockBytes, 2 * kTcBlockBytes,
                 &full[s]);
        last_phase[s] = (long)(g / kPStages);
      }
    }
  } else if (warp == 1 && lane == 0) {
    uint32_t g = 0, u = 0;
    for (long t = blockIdx.x; t < ntot && !*(volatile int *)&abort_flag; t += gridDim.x) {
      const TcArgs *A;
      long i0, j0;
      if (!tile(t, A, i0, j0)) continue;
      const uint32_t b = u & 1;
      if (u >= 2 && !mbar_wait(&acce[b], ((u / 2) - 1) & 1, lim)) {
        atomicExch(&abort_flag, 1);
        break;
      }
      tc_fence_after();
      const uint32_t acc = tmem + b * 256;
      bool ok = true;
      for (long k = 0; k < A->KS; k++, g++) {
        const int s = (int)(g % kPStages);
        if (!mbar_wait(&full[s], (g / kPStages) & 1, lim)) {
          ok = false;
          break;
        }
        tc_fence_after();
        const uint32_t sa = smem_u32(ring + (size_t)s * kTcStageBytes), sb = sa + kTcBlockBytes;
#pragma unroll
        for (int kk = 0; kk < kTcStageK / 32; kk++)
          umma_i8(acc, umma_desc(sa + kk * 256, 128, 1024), umma_desc(sb + kk * 256, 128, 1024),
                  (k > 0 || kk > 0) ? 1u : 0u);
        umma_commit(&empty[s]);
      }
      if (!ok) {
        atomicExch(&abort_flag, 1);
        break;
      }
      umma_commit(&accf[b]);
      u++;
    }
    umma_commit(&done);  // arrives when every MMA issued above has completed
  } else if (warp >= 2) {
    const int q = warp & 3;                // tensor-memory lane quarter this warp may read
    const int half = (warp - 2) >> 2;      // which half of the accumulator's columns it reads
    uint32_t u = 0;
    for (long t = blockIdx.x; t < ntot; t += gridDim.x) {
      const int stop = __shfl_sync(0xffffffffu, lane == 0 ? *(volatile int *)&abort_flag : 0, 0);
      if (stop) break;
      const TcArgs *A;
      long i0, j0;
      if (!tile(t, A, i0, j0)) continue;
      const uint32_t b = u & 1;
      const bool ok = __all_sync(0xffffffffu, mbar_wait(&accf[b], (u / 2) & 1, lim));
      if (!ok) {
        if (lane == 0) atomicExch(&abort_flag, 1);
        break;
      }
      tc_fence_after();
      tc_tile_epilogue(*A, i0, j0, tmem + b * 256, q, lane, half * 8, 8);
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(&acce[b]);
      u++;
    }
  }
  __syncwarp();
  __syncthreads();
  // Every MMA this CTA issued has completed once `done` arrives (the issuer commits it on every path); after a
  // timeout, the last fill of each stage also lands before the ring is released.
  if (threadIdx.x == 0) {
    if (*(volatile int *)&abort_flag) {
      atomicAdd(ga.err, 1ull);
      for (int s = 0; s < kPStages; s++)
        if (last_phase[s] >= 0) mbar_wait(&full[s], (uint32_t)(last_phase[s] & 1), lim);
    }
    mbar_wait(&done, 0, lim);
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(512u));
}

}  // namespace tn93
