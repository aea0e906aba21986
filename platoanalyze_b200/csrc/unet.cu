// Learned warm start: a 3-level 3D U-Net (16-32-64 channels) on the nodes of a box mesh,
// trained and evaluated with hand-written BF16 tensor-core kernels (no reference
// counterpart: Plato Analyze has no learned component).
//
// Tensors are channels-last (b, d, h, w, c) with a one-voxel zero halo on every side, so a
// 3x3x3 convolution with zero padding reads its neighbours without bounds checks; kernels
// only ever write interior voxels.  Activations are BF16, activation gradients FP32,
// parameters FP32 (Adam) with BF16 copies for the tensor cores.
//
//  * Convolution (forward and data gradient): implicit GEMM, M = voxels, N = output
//    channels, K = taps x input channels, mma.sync.m16n8k16 BF16 -> FP32; each warp owns
//    32 voxels x all output channels; A fragments are gathered straight from the haloed
//    tensor (pairs of channels are 32-bit words), B fragments from the weights laid out
//    [tap][out][in].  Bias, ReLU and FP32 accumulation are fused in the epilogue.  The data
//    gradient is the same convolution with flipped, transposed weights.
//  * Weight gradient: GEMM over voxels, M = output channels, N = input channels, K =
//    voxels; a CTA stages 64-voxel tiles of the masked output gradient and of the shifted
//    input in shared memory and feeds the tensor cores with ldmatrix.trans; partial sums
//    are added to the FP32 gradient with atomics.
//  * 2x2x2 average pooling, nearest upsampling, the ReLU gradient mask, the loss and Adam
//    are element-wise kernels.
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

#include "plato_b200.h"

namespace {

using bf16 = __nv_bfloat16;

std::string g_unet_error;

int fail(int status, const std::string& msg) {
    g_unet_error = msg;
    return status;
}

#define UCUDA(expr)                                                                               \
    do {                                                                                          \
        cudaError_t _e = (expr);                                                                  \
        if (_e != cudaSuccess) {                                                                  \
            (void)cudaGetLastError();                                                             \
            return fail(_e == cudaErrorMemoryAllocation ? PLATO_OUT_OF_MEMORY : PLATO_CUDA_ERROR, \
                        std::string("CUDA error ") + cudaGetErrorName(_e) + " in " #expr);        \
        }                                                                                         \
    } while (0)

#define ULAUNCH()                                                                              \
    do {                                                                                       \
        cudaError_t _e = cudaGetLastError();                                                   \
        if (_e != cudaSuccess)                                                                 \
            return fail(PLATO_CUDA_ERROR, std::string("kernel launch failed: ") + cudaGetErrorName(_e)); \
    } while (0)

// A channel slice [c0, c0 + C) of a haloed channels-last tensor with ld channels per voxel.
struct TView {
    void*   p;
    int32_t ld, c0;
    int32_t B, D, H, W;  // interior extents
};

__host__ __device__ __forceinline__ int64_t halo_index(const TView& t, int64_t v) {
    const int64_t x = v % t.W;
    int64_t r = v / t.W;
    const int64_t y = r % t.H;
    r /= t.H;
    const int64_t z = r % t.D;
    const int64_t b = r / t.D;
    return ((b * (t.D + 2) + z + 1) * (t.H + 2) + y + 1) * (t.W + 2) + x + 1;
}

// voxel coordinates of plain interior index v of a view, and the haloed position of a voxel, in
// 32-bit arithmetic (a network's grids hold fewer than 2^31 positions, checked at creation)
struct Vox {
    int b, z, y, x;
};
__device__ __forceinline__ Vox vox_of(const TView& t, uint32_t v) {
    Vox r;
    r.x = int(v % uint32_t(t.W));
    v /= uint32_t(t.W);
    r.y = int(v % uint32_t(t.H));
    v /= uint32_t(t.H);
    r.z = int(v % uint32_t(t.D));
    r.b = int(v / uint32_t(t.D));
    return r;
}
__device__ __forceinline__ int32_t hpos(const TView& t, int b, int z, int y, int x) {
    return ((b * (t.D + 2) + z + 1) * (t.H + 2) + y + 1) * (t.W + 2) + x + 1;
}

__device__ __forceinline__ void mma16816(float (&c)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

__device__ __forceinline__ uint32_t ld32(const bf16* p) { return *reinterpret_cast<const uint32_t*>(p); }

__device__ __forceinline__ uint32_t pack_bf16(float a, float b) {
    __nv_bfloat162 v = __floats2bfloat162_rn(a, b);
    return *reinterpret_cast<uint32_t*>(&v);
}

// ---- convolution: forward and data gradient ---------------------------------------------
// out[v][co] (+)= act(bias[co] + sum_t sum_ci W[t][co][ci] in[v + o_t][ci]); TAPS = 27
// (3x3x3, zero padding) or 1.  COUTP = COUT rounded up to 8 (weights padded with zeros).
constexpr int kConvWarps = 4;
constexpr int kMT = 2;  // 16-voxel m-tiles per warp

template <int CIN, int COUT, int TAPS, bool RELU, bool OUT_F32, bool ACCUM>
__global__ void __launch_bounds__(kConvWarps * 32)
k_conv(TView in, const bf16* __restrict__ Wt, const float* __restrict__ bias, TView out, int64_t nvox) {
    static_assert(CIN % 16 == 0, "input channels must be a multiple of 16");
    constexpr int COUTP = (COUT + 7) / 8 * 8;
    constexpr int NT = COUTP / 8;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int g = lane >> 2, tig = lane & 3;
    const int64_t vbase = (int64_t(blockIdx.x) * kConvWarps + warp) * (16 * kMT);
    if (vbase >= nvox) return;
    const bf16* __restrict__ ip = static_cast<const bf16*>(in.p);
    // haloed voxel offsets of the rows this lane touches (rows g and g+8 of each m-tile)
    int64_t rowoff[kMT][2];
    bool rowok[kMT][2];
#pragma unroll
    for (int m = 0; m < kMT; ++m)
#pragma unroll
        for (int hlf = 0; hlf < 2; ++hlf) {
            const int64_t v = vbase + 16 * m + g + 8 * hlf;
            rowok[m][hlf] = v < nvox;
            rowoff[m][hlf] = (rowok[m][hlf] ? halo_index(in, v) : 0) * in.ld + in.c0 + 2 * tig;
        }
    float acc[kMT][NT][4];
#pragma unroll
    for (int m = 0; m < kMT; ++m)
#pragma unroll
        for (int n = 0; n < NT; ++n)
#pragma unroll
            for (int q = 0; q < 4; ++q) acc[m][n][q] = 0.f;
    const int64_t sy = in.W + 2, sz = int64_t(in.H + 2) * (in.W + 2);
    for (int t = 0; t < TAPS; ++t) {
        int64_t o = 0;
        if (TAPS == 27) o = ((t / 9 - 1) * sz + ((t / 3) % 3 - 1) * sy + (t % 3 - 1)) * in.ld;
        const bf16* __restrict__ wt = Wt + int64_t(t) * COUTP * CIN;
#pragma unroll
        for (int kc = 0; kc < CIN / 16; ++kc) {
            uint32_t a[kMT][4];
#pragma unroll
            for (int m = 0; m < kMT; ++m) {
                const bf16* r0 = ip + rowoff[m][0] + o + 16 * kc;
                const bf16* r1 = ip + rowoff[m][1] + o + 16 * kc;
                a[m][0] = rowok[m][0] ? ld32(r0) : 0u;
                a[m][1] = rowok[m][1] ? ld32(r1) : 0u;
                a[m][2] = rowok[m][0] ? ld32(r0 + 8) : 0u;
                a[m][3] = rowok[m][1] ? ld32(r1 + 8) : 0u;
            }
#pragma unroll
            for (int n = 0; n < NT; ++n) {
                const bf16* wp = wt + (8 * n + g) * CIN + 16 * kc + 2 * tig;
                const uint32_t b0 = ld32(wp), b1 = ld32(wp + 8);
#pragma unroll
                for (int m = 0; m < kMT; ++m) mma16816(acc[m][n], a[m], b0, b1);
            }
        }
    }
    // epilogue: rows g / g+8, columns 8n + 2 tig + {0, 1}
#pragma unroll
    for (int m = 0; m < kMT; ++m)
#pragma unroll
        for (int hlf = 0; hlf < 2; ++hlf) {
            const int64_t v = vbase + 16 * m + g + 8 * hlf;
            if (v >= nvox) continue;
            const int64_t base = halo_index(out, v) * out.ld + out.c0;
#pragma unroll
            for (int n = 0; n < NT; ++n) {
                const int c = 8 * n + 2 * tig;
                if (c >= COUT) continue;
                float y0 = acc[m][n][2 * hlf], y1 = acc[m][n][2 * hlf + 1];
                if (bias) {
                    y0 += bias[c];
                    if (c + 1 < COUT) y1 += bias[c + 1];
                }
                if (RELU) {
                    y0 = fmaxf(y0, 0.f);
                    y1 = fmaxf(y1, 0.f);
                }
                if (OUT_F32) {
                    float* op = static_cast<float*>(out.p) + base + c;
                    if (ACCUM) {
                        op[0] += y0;
                        if (c + 1 < COUT) op[1] += y1;
                    } else {
                        op[0] = y0;
                        if (c + 1 < COUT) op[1] = y1;
                    }
                } else {
                    *reinterpret_cast<uint32_t*>(static_cast<bf16*>(out.p) + base + c) = pack_bf16(y0, y1);
                }
            }
        }
}

// ---- convolution on the 5th-generation tensor cores (tcgen05, TMEM accumulator) -----------
// The same implicit GEMM as k_conv, tiled over HALOED positions: a tile is 128 consecutive
// positions p0 .. p0 + 127 of the zero-haloed channels-last input (UMMA M = 128) with every output
// channel (N = COUTP, a multiple of 16); its FP32 accumulator lives in tensor memory, 128 lanes x
// N columns.  Tap (dz, dy, dx) of output row m reads the input at position p0 + m + dz sz +
// dy sy + dx (sy = W + 2, sz = (H + 2) sy), so for one dz the 9 taps' A operands are 128-row
// windows, dy sy + dx rows apart, of ONE slab of 128 + 2 (sy + 1) consecutive input rows.  All
// threads copy a slab with cp.async (16 bytes = 8 channels, zero fill outside the tensor) into
// the canonical K-major, no-swizzle layout (core matrices of 8 rows x 16 bytes: row r of K-chunk
// c at c * LBO + r * 16, so a window starting at any row is again such a matrix) -- or, with 16
// input channels, rows of 32 bytes in the 32-byte swizzle (2.7 % faster forward); one thread then
// issues 9 x CIN / 16 tcgen05.mma (kind::f16: BF16 A and B, FP32 accumulate) whose A descriptors
// start at the tap's row and commits them to the buffer's mbarrier: 3 slabs per tile instead of
// 27 gathered tap tiles.  The CTAs are persistent (tile = blockIdx.x + k gridDim.x): every tap's
// weights stay in shared memory when they fit (else each buffer carries its slab's 9 taps), the
// slabs run through 2 to 4 buffers with later slabs' copies in flight while the tensor core works,
// and two accumulators alternate so that tile k - 1's epilogue runs after tile k's first MMAs are
// queued.  A 1x1x1 convolution is one slab of 128 rows per tile.  Outputs at halo positions are
// computed and discarded.  The epilogue loads an accumulator with tcgen05.ld (warp w reads TMEM
// lanes 32w .. 32w + 31, the rows of its 32 positions), adds the bias, applies ReLU and stores
// the interior positions.  Every mbarrier wait is bounded: on a timeout the CTA stops issuing,
// waits (bounded) for what it issued, raises *err, skips the stores and still frees its tensor
// memory.  With 16 output channels an MMA (128 x 16 x 16) reads a 4 KB A window for 512 B of
// weights; these layers take about 50 cycles per MMA with the unswizzled operands.
constexpr int kTcRows = 128;             // haloed positions per CTA (UMMA M)
constexpr uint32_t kTcPolls = 1u << 22;  // bounded mbarrier polls (about half a second)

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// shared-memory matrix descriptor: K-major, no swizzle; start, leading (K) and stride (M/N)
// byte offsets in 16-byte units, descriptor version 1 (bits 46-47)
__device__ __forceinline__ uint64_t umma_smem_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    return uint64_t((saddr >> 4) & 0x3FFFu) | (uint64_t((lbo >> 4) & 0x3FFFu) << 16) |
           (uint64_t((sbo >> 4) & 0x3FFFu) << 32) | (uint64_t(1) << 46);
}

// K-major SWIZZLE_32B descriptor (layout type 6 at bits 61-63) of a 16-channel slab window: rows
// of 32 bytes, 8-row groups 256 B apart (stride offset), leading offset 16 B (unused within
// the swizzle width), base offset 0.  The data is stored with its 16-byte chunk index XOR bit 7
// of the row's shared-memory address, so a window may start at any row.  (Measured: with the
// base offset set from the start address instead, the products came out wrong.)
__device__ __forceinline__ uint64_t umma_smem_desc_sw32(uint32_t saddr) {
    return uint64_t((saddr >> 4) & 0x3FFFu) | (uint64_t(1) << 16) | (uint64_t(256 >> 4) << 32) | (uint64_t(1) << 46) |
           (uint64_t(6) << 61);
}

// instruction descriptor of kind::f16: FP32 accumulator (bits 4-5 = 1), BF16 A and B (bits
// 7-9, 10-12 = 1), both K-major, N >> 3 at bits 17-22, M >> 4 at bits 24-28
template <int N>
__host__ __device__ constexpr uint32_t umma_idesc_bf16_f32() {
    return (1u << 4) | (1u << 7) | (1u << 10) | (uint32_t(N >> 3) << 17) | (uint32_t(kTcRows >> 4) << 24);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

// waits for the completion of the phase with the given parity; false when the poll bound ran out
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
    const uint32_t a = smem_u32(bar);
    for (uint32_t i = 0; i < kTcPolls; ++i) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.b32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(a), "r"(parity)
            : "memory");
        if (done) return true;
        __nanosleep(64);
    }
    return false;
}

__device__ __forceinline__ void cp_async16(uint32_t dst, const void* src, uint32_t src_bytes) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(src_bytes) : "memory");
}

__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
        "l"(da), "l"(db), "r"(idesc), "r"(acc)
        : "memory");
}

__device__ __forceinline__ void umma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&r)[16]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr)
        : "memory");
}

template <int COUTP>
constexpr int tc_tmem_cols() {
    return COUTP <= 32 ? 32 : (COUTP <= 64 ? 64 : (COUTP <= 128 ? 128 : 256));
}

// Row stride of a staged slab: at least its rows, chosen modulo 8 so that the 16-byte chunks
// that 8 consecutive threads copy (a row's CIN / 8 chunks, then the next row's) fall in distinct
// 128-byte bank groups.
inline int tc_row_stride(int nrows, int cin8) {
    const int want = cin8 == 2 ? 4 : (cin8 == 4 ? 2 : 7);
    return nrows + ((want - nrows % 8) + 8) % 8;
}

// Launch geometry of k_conv_tc, chosen on the host.  Positions are haloed indices of the input
// (and output) grid, below 2^31.
struct TcGeom {
    int32_t pfirst, plast, ptotal;  // first and last interior position, all positions
    int32_t ntiles;                 // 128-position tiles from pfirst to plast
    int32_t rows;                   // slab row stride (>= the rows one slab gathers)
    int32_t nbuf;                   // slab buffers in the pipeline (2 to 4)
    int32_t lag;                    // MMAs of slab i issued in iteration i + lag (1 <= lag < nbuf)
    int32_t wres;                   // 1: all taps' weights stay in shared memory; 0: staged per slab
    uint32_t w_bytes;               // shared memory of the resident weights (0 when staged)
    uint32_t buf_bytes;             // one slab buffer (with its taps' weights when staged)
};

template <int CIN, int COUT, int TAPS, bool RELU, bool OUT_F32, bool ACCUM>
__global__ void __launch_bounds__(128)
k_conv_tc(TView in, const bf16* __restrict__ Wt, const float* __restrict__ bias, TView out, TcGeom g,
          int* __restrict__ err) {
    constexpr int COUTP = (COUT + 15) / 16 * 16;
    static_assert(CIN % 16 == 0 && COUTP <= 256, "UMMA shape");
    constexpr int NDZ = TAPS == 27 ? 3 : 1, TPD = TAPS / NDZ;  // slabs (z offsets) per tile, taps per slab
    constexpr bool SW = CIN == 16;  // 16-channel slabs: rows of 32 B in the 32-byte swizzle
    constexpr int ACC_COLS = tc_tmem_cols<COUTP>();            // one accumulator; two are allocated
    constexpr uint32_t BTAP = uint32_t(COUTP) * CIN * 2;       // one tap's weights
    constexpr uint32_t LBO_B = (COUTP / 8) * 128;
    constexpr uint32_t IDESC = umma_idesc_bf16_f32<COUTP>();
    const uint32_t LBO_A = uint32_t(g.rows) * 16u;  // bytes between the 8-channel chunks of a slab row
    const uint32_t A_BYTES = uint32_t(g.rows) * CIN * 2;
    extern __shared__ __align__(128) uint8_t tc_smem[];
    // mbarriers: MMA completion per slab buffer (4), per accumulator (2), all MMAs (1)
    __shared__ __align__(8) uint64_t bar[7];
    __shared__ uint32_t tmem_slot;
    __shared__ float sbias[COUTP];
    const int tid = threadIdx.x, warp = tid >> 5;
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_slot)),
                     "r"(2 * ACC_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0) {
        for (int q = 0; q < 7; ++q) mbar_init(&bar[q], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    for (int c = tid; c < COUTP; c += 128) sbias[c] = (bias && c < COUT) ? bias[c] : 0.f;
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = tmem_slot;
    const int32_t sy = in.W + 2, sz = (in.H + 2) * sy;
    const int halo = TAPS == 27 ? sy + 1 : 0;
    const int nrows = kTcRows + 2 * halo;  // slab rows gathered
    const int nbuf = g.nbuf, lag = g.lag;
    const int my_tiles = (g.ntiles - int(blockIdx.x) + int(gridDim.x) - 1) / int(gridDim.x);
    const int nslabs = my_tiles * NDZ;
    const bf16* __restrict__ ip = static_cast<const bf16*>(in.p);
    const uint32_t sbase = smem_u32(tc_smem), wbase = sbase, bbase = sbase + g.w_bytes;

    // epilogue of the k-th tile of this CTA from accumulator k & 1: bias, ReLU, store the
    // interior positions (all threads; thread t owns TMEM lane t = the tile's row t)
    auto epilogue = [&](int k) {
        const int32_t p = g.pfirst + (int(blockIdx.x) + k * int(gridDim.x)) * kTcRows + tid;
        bool row_ok = p <= g.plast;
        if (row_ok) {
            uint32_t t = uint32_t(p);
            const uint32_t x = t % uint32_t(sy);
            t /= uint32_t(sy);
            const uint32_t y = t % uint32_t(in.H + 2);
            t /= uint32_t(in.H + 2);
            const uint32_t z = t % uint32_t(in.D + 2);
            row_ok = x >= 1u && x <= uint32_t(in.W) && y >= 1u && y <= uint32_t(in.H) && z >= 1u && z <= uint32_t(in.D);
        }
        const int64_t obase = int64_t(p) * out.ld + out.c0;
        const uint32_t acc = tmem + (uint32_t(32 * warp) << 16) + uint32_t((k & 1) * ACC_COLS);
#pragma unroll
        for (int c0 = 0; c0 < COUTP; c0 += 16) {
            uint32_t r[16];
            tmem_ld16(acc + uint32_t(c0), r);
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            if (!row_ok) continue;
            float y[16];
#pragma unroll
            for (int j = 0; j < 16; ++j) {
                y[j] = __uint_as_float(r[j]) + sbias[c0 + j];
                if (RELU) y[j] = fmaxf(y[j], 0.f);
            }
            if (OUT_F32) {
                float* op = static_cast<float*>(out.p) + obase + c0;
                if (c0 + 16 <= COUT) {
#pragma unroll
                    for (int j = 0; j < 16; j += 4) {
                        float4 w4 = make_float4(y[j], y[j + 1], y[j + 2], y[j + 3]);
                        if (ACCUM) {
                            const float4 o4 = *reinterpret_cast<const float4*>(op + j);
                            w4.x += o4.x; w4.y += o4.y; w4.z += o4.z; w4.w += o4.w;
                        }
                        *reinterpret_cast<float4*>(op + j) = w4;
                    }
                } else {
#pragma unroll
                    for (int j = 0; j < 16; ++j)
                        if (c0 + j < COUT) op[j] = ACCUM ? op[j] + y[j] : y[j];
                }
            } else {
                bf16* op = static_cast<bf16*>(out.p) + obase + c0;
                if (c0 + 16 <= COUT) {
                    uint4 lo, hi;
                    lo.x = pack_bf16(y[0], y[1]); lo.y = pack_bf16(y[2], y[3]);
                    lo.z = pack_bf16(y[4], y[5]); lo.w = pack_bf16(y[6], y[7]);
                    hi.x = pack_bf16(y[8], y[9]); hi.y = pack_bf16(y[10], y[11]);
                    hi.z = pack_bf16(y[12], y[13]); hi.w = pack_bf16(y[14], y[15]);
                    reinterpret_cast<uint4*>(op)[0] = lo;
                    reinterpret_cast<uint4*>(op)[1] = hi;
                } else {
#pragma unroll
                    for (int j = 0; j < 16; ++j)
                        if (c0 + j < COUT) op[j] = __float2bfloat16_rn(y[j]);
                }
            }
        }
        // the accumulator is rewritten two tiles later, by MMAs issued after a barrier
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    };

    bool ok = true;
    int issued = 0;
    // iteration i copies slab i (tile i / NDZ of this CTA, z offset i % NDZ - 1) into buffer
    // i % nbuf and issues the MMAs of slab i - lag (lag < nbuf); a buffer is refilled once the
    // MMAs of the slab it held, issued in iteration i - nbuf + lag, have completed
    for (int i = 0; i < nslabs + lag; ++i) {
        if (i < nslabs) {
            const int b = i % nbuf;
            if (i >= nbuf) {
                bool w = true;
                if (tid == 0) w = mbar_wait(&bar[b], uint32_t((i - nbuf) / nbuf) & 1u);
                ok = __syncthreads_and(w) != 0;
                if (!ok) break;
            }
            const int k = i / NDZ, dzi = i - k * NDZ;
            const int32_t p0 = g.pfirst + (int(blockIdx.x) + k * int(gridDim.x)) * kTcRows;
            const int32_t r0 = p0 + (NDZ == 3 ? (dzi - 1) * sz : 0) - halo;  // position of slab row 0
            const uint32_t a_s = bbase + uint32_t(b) * g.buf_bytes;
            for (int q = tid; q < nrows * (CIN / 8); q += 128) {  // consecutive threads: one row's chunks
                const int r = q / (CIN / 8), c8 = q - r * (CIN / 8);
                const int32_t pos = r0 + r;
                const bool inside = pos >= 0 && pos < g.ptotal;  // rows outside feed discarded outputs only
                uint32_t dst = a_s + uint32_t(c8) * LBO_A + uint32_t(r) * 16u;
                if (SW) {
                    const uint32_t row = a_s + 32u * uint32_t(r);
                    dst = row + 16u * (uint32_t(c8) ^ ((row >> 7) & 1u));
                }
                cp_async16(dst, inside ? ip + int64_t(pos) * in.ld + in.c0 + 8 * c8 : ip, inside ? 16u : 0u);
            }
            // weights [tap][COUTP][CIN]: every tap once (resident), or this slab's taps per buffer
            const int wt0 = g.wres ? 0 : dzi * TPD, nw = g.wres ? (i == 0 ? TAPS : 0) : TPD;
            const uint32_t w_s = g.wres ? wbase : a_s + A_BYTES;
            for (int q = tid; q < nw * COUTP * (CIN / 8); q += 128) {
                const int j = q / (COUTP * (CIN / 8)), rem = q - j * (COUTP * (CIN / 8));
                const int n = rem / (CIN / 8), c8 = rem - n * (CIN / 8);
                cp_async16(w_s + uint32_t(j) * BTAP + uint32_t(c8) * LBO_B + uint32_t(n >> 3) * 128u + uint32_t(n & 7) * 16u,
                           Wt + (int64_t(wt0 + j) * COUTP + n) * CIN + 8 * c8, 16u);
            }
        }
        asm volatile("cp.async.commit_group;" ::: "memory");  // one group per iteration (empty past the last slab)
        if (i >= lag) {
            const int s = i - lag, b = s % nbuf, k = s / NDZ, dzi = s - k * NDZ;
            // slab s is in; the lag - 1 later ones may still be in flight
            if (lag == 1) asm volatile("cp.async.wait_group 0;" ::: "memory");
            else if (lag == 2) asm volatile("cp.async.wait_group 1;" ::: "memory");
            else asm volatile("cp.async.wait_group 2;" ::: "memory");
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // visible to the tensor core
            __syncthreads();
            if (tid == 0) {
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                const uint32_t a_s = bbase + uint32_t(b) * g.buf_bytes;
                const uint32_t w_s = g.wres ? wbase + uint32_t(dzi * TPD) * BTAP : a_s + A_BYTES;
                const uint32_t d = tmem + uint32_t((k & 1) * ACC_COLS);
#pragma unroll 1
                for (int j = 0; j < TPD; ++j) {
                    // tap (dz, dy, dx): its 128 rows start dy sy + dx rows from the slab's centre window
                    const int dy = TPD == 9 ? j / 3 - 1 : 0, dx = TPD == 9 ? j % 3 - 1 : 0;
                    const uint32_t a_t = a_s + uint32_t(halo + dy * sy + dx) * (SW ? 32u : 16u);
#pragma unroll
                    for (int kc = 0; kc < CIN / 16; ++kc)
                        umma_bf16(d, SW ? umma_smem_desc_sw32(a_t) : umma_smem_desc(a_t + 2u * kc * LBO_A, LBO_A, 128u),
                                  umma_smem_desc(w_s + uint32_t(j) * BTAP + 2u * kc * LBO_B, LBO_B, 128u), IDESC,
                                  (dzi > 0 || j > 0 || kc > 0) ? 1u : 0u);
                }
                umma_commit(&bar[b]);
                if (dzi == NDZ - 1) umma_commit(&bar[4 + (k & 1)]);  // tile k's accumulator is complete
            }
            ++issued;
            if (dzi == 0 && k >= 1) {  // tile k's first MMAs are queued: store tile k - 1 meanwhile
                bool w = true;
                if (tid == 0) w = mbar_wait(&bar[4 + ((k - 1) & 1)], uint32_t((k - 1) >> 1) & 1u);
                ok = __syncthreads_and(w) != 0;
                if (!ok) break;
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                epilogue(k - 1);
            }
        }
    }
    asm volatile("cp.async.wait_all;" ::: "memory");  // no copy into shared memory outlives the loop
    // all issued MMAs complete (bounded even after a timeout above)
    bool fin = true;
    if (tid == 0) {
        if (issued > 0) umma_commit(&bar[6]);
        fin = issued == 0 || mbar_wait(&bar[6], 0u);
    }
    const bool good = __syncthreads_and(ok && fin) != 0;
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (good) {
        if (my_tiles > 0) epilogue(my_tiles - 1);
    } else if (tid == 0) {
        atomicExch(err, 1);
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(2 * ACC_COLS) : "memory");
}

// ---- weight gradient --------------------------------------------------------------------
// dW[t][co][ci] += sum_p dy[p][co] x[p + o_t][ci] over the interior haloed positions p (dy is
// read as zero elsewhere; x's halo holds zeros).  Grid (CTAs per tap group, G tap groups): a CTA
// owns TAPS / G consecutive taps and loops over 128-position tiles (tile = blockIdx.x + k gridDim.x).
// Per tile it stages the tile's dy rows and, per z offset of its taps, one slab of x rows that
// every tap of that z offset reads at a shifted row (cp.async, double-buffered: the next tile's
// copies are in flight while this tile's MMAs run).  Warps own output tiles (tap, 16 co, 8 ci)
// and keep their sums in registers over all of the CTA's tiles: mma.sync m16n8k16 with A = dy^T
// and B = x, both through ldmatrix.trans (one A fragment per k-step serves every tap).  One
// atomic add per output element and CTA at the end.  (The tensor-core MMA of tcgen05 needs M >= 64
// rows of one operand at a uniform shared-memory stride; here M is 16 output channels, and the
// taps that would fill it read the slab at non-uniform shifts.)
constexpr int kWgRows = 128;  // positions per tile (8 k-steps)

__device__ __forceinline__ void ldsm_x4_t(uint32_t (&r)[4], const bf16* p) {
    const uint32_t a = static_cast<uint32_t>(__cvta_generic_to_shared(p));
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0,%1,%2,%3}, [%4];\n"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
                 : "r"(a));
}
__device__ __forceinline__ void ldsm_x2_t(uint32_t& r0, uint32_t& r1, const bf16* p) {
    const uint32_t a = static_cast<uint32_t>(__cvta_generic_to_shared(p));
    asm volatile("ldmatrix.sync.aligned.m8n8.x2.trans.shared.b16 {%0,%1}, [%2];\n" : "=r"(r0), "=r"(r1) : "r"(a));
}

// tap groups of a weight-gradient launch: the fewest (1, 3, 9 or 27) that leave each warp at most
// 18 output tiles (72 FP32 sums in registers)
template <int CIN, int COUT, int TAPS>
constexpr int wg_groups() {
    if (TAPS == 1) return 1;
    constexpr int per_tap = (COUT / 16) * (CIN / 8);
    return (27 * per_tap + 3) / 4 <= 18 ? 1 : (9 * per_tap + 3) / 4 <= 18 ? 3 : (3 * per_tap + 3) / 4 <= 18 ? 9 : 27;
}

// offset of tap t of a 3x3x3 stencil in haloed positions
__host__ __device__ __forceinline__ int wg_tap_offset(int t, int sy, int sz) {
    return (t / 9 - 1) * sz + ((t / 3) % 3 - 1) * sy + (t % 3 - 1);
}

// half-width (rows) of the x slab of a tap group: all 9 taps of a z offset, 3 taps of a row, one tap
template <int TAPS, int G>
__host__ __device__ __forceinline__ int wg_halfwidth(int sy) {
    return TAPS == 1 ? 0 : (G <= 3 ? sy + 1 : (G == 9 ? 1 : 0));
}

template <int CIN, int COUT, int TAPS, int G>
__global__ void __launch_bounds__(128)
k_conv_wgrad(TView x, TView dy, float* __restrict__ dW, int cout_real, int32_t pfirst, int32_t plast, int32_t ptotal,
             int32_t ntiles, int rows_pad, uint32_t stage_elems) {
    static_assert(COUT % 16 == 0 && CIN % 16 == 0, "channel counts");
    constexpr int TPG = TAPS / G;                         // taps of this CTA
    constexpr int NSL = (TAPS == 27 && G == 1) ? 3 : 1;   // x slabs per tile (one per z offset)
    constexpr int LDY = COUT + 8, LDX = CIN + 8;          // padded rows: 16-byte aligned, no ldmatrix conflicts
    constexpr int T = TPG * (COUT / 16) * (CIN / 8);      // output tiles of 16 x 8
    // with at most two output tiles (the 1x1x1 head), pairs of warps share a tile and split its
    // k-steps (even / odd), so all four warps work; each adds its own partial sums
    constexpr int KSPLIT = T <= 2 ? 2 : 1;
    constexpr int WPT = 4 / KSPLIT;
    constexpr int PER = (T + WPT - 1) / WPT;
    extern __shared__ __align__(16) bf16 wg_smem[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int wt = warp % WPT, kg = warp / WPT;
    const int g = blockIdx.y;
    const int32_t sy = x.W + 2, sz = (x.H + 2) * sy;
    const int hw = wg_halfwidth<TAPS, G>(sy);
    const int srows = kWgRows + 2 * hw;  // rows of one slab (rows_pad >= srows is their stride)
    // slab centre offsets: the middle tap of each z offset (G = 1), else of the group
    int32_t centre[NSL];
#pragma unroll
    for (int sl = 0; sl < NSL; ++sl)
        centre[sl] = TAPS == 1 ? 0 : wg_tap_offset(NSL == 3 ? 9 * sl + 4 : g * TPG + TPG / 2, sy, sz);
    // this warp's output tiles: element offset of its B rows (k-step 0, lane's row) and its A block
    int boff[PER], mtile[PER];
#pragma unroll
    for (int k = 0; k < PER; ++k) {
        const int id = wt + WPT * k;
        const int j = id / ((COUT / 16) * (CIN / 8)), rem = id - j * ((COUT / 16) * (CIN / 8));
        const int mt = rem / (CIN / 8), nt = rem - mt * (CIN / 8);
        const int sl = NSL == 3 ? j / 9 : 0;
        const int rel = TAPS == 1 ? 0 : wg_tap_offset(g * TPG + j, sy, sz) - centre[sl];
        boff[k] = (kWgRows * LDY) + (sl * rows_pad + hw + rel + (lane & 7) + ((lane >> 3) & 1) * 8) * LDX + 8 * nt;
        mtile[k] = mt;
    }
    float acc[PER][4];
#pragma unroll
    for (int k = 0; k < PER; ++k)
#pragma unroll
        for (int q = 0; q < 4; ++q) acc[k][q] = 0.f;
    const bf16* __restrict__ yp = static_cast<const bf16*>(dy.p);
    const bf16* __restrict__ xp = static_cast<const bf16*>(x.p);
    const int my_tiles = (ntiles - int(blockIdx.x) + int(gridDim.x) - 1) / int(gridDim.x);
    const uint32_t sbase = static_cast<uint32_t>(__cvta_generic_to_shared(wg_smem));

    // copies of tile k into stage buf: dy rows (zero outside the interior), then the x slabs
    auto stage = [&](int k, int buf) {
        const int32_t p0 = pfirst + (int(blockIdx.x) + k * int(gridDim.x)) * kWgRows;
        const uint32_t st = sbase + uint32_t(buf) * stage_elems * 2u;
        for (int q = threadIdx.x; q < kWgRows * (COUT / 8); q += 128) {
            const int r = q / (COUT / 8), c8 = q - r * (COUT / 8);
            const int32_t p = p0 + r;
            bool in = p <= plast;
            if (in) {
                uint32_t t = uint32_t(p);
                const uint32_t xx = t % uint32_t(sy);
                t /= uint32_t(sy);
                const uint32_t yy = t % uint32_t(x.H + 2);
                t /= uint32_t(x.H + 2);
                const uint32_t zz = t % uint32_t(x.D + 2);
                in = xx >= 1u && xx <= uint32_t(x.W) && yy >= 1u && yy <= uint32_t(x.H) && zz >= 1u && zz <= uint32_t(x.D);
            }
            cp_async16(st + uint32_t(r * LDY + 8 * c8) * 2u, in ? yp + int64_t(p) * dy.ld + dy.c0 + 8 * c8 : yp,
                       in ? 16u : 0u);
        }
#pragma unroll
        for (int sl = 0; sl < NSL; ++sl) {
            const int32_t r0 = p0 + centre[sl] - hw;
            const uint32_t xs = st + uint32_t(kWgRows * LDY + sl * rows_pad * LDX) * 2u;
            for (int q = threadIdx.x; q < srows * (CIN / 8); q += 128) {
                const int r = q / (CIN / 8), c8 = q - r * (CIN / 8);
                const int32_t pos = r0 + r;
                const bool in = pos >= 0 && pos < ptotal;
                cp_async16(xs + uint32_t(r * LDX + 8 * c8) * 2u, in ? xp + int64_t(pos) * x.ld + x.c0 + 8 * c8 : xp,
                           in ? 16u : 0u);
            }
        }
    };

    if (my_tiles > 0) stage(0, 0);
    asm volatile("cp.async.commit_group;" ::: "memory");
    for (int k = 0; k < my_tiles; ++k) {
        if (k + 1 < my_tiles) stage(k + 1, (k + 1) & 1);
        asm volatile("cp.async.commit_group;" ::: "memory");
        asm volatile("cp.async.wait_group 1;" ::: "memory");  // tile k is in; tile k + 1 may be in flight
        __syncthreads();
        const bf16* sb = wg_smem + size_t(k & 1) * stage_elems;
#pragma unroll
        for (int ks = 0; ks < kWgRows / 16; ++ks) {
            if (ks % KSPLIT != kg) continue;
            // A = dy^T (rows co, cols position): matrices (m0, k0), (m0+8, k0), (m0, k0+8), (m0+8, k0+8)
            uint32_t a[COUT / 16][4];
            const int mat = lane >> 3, rr = lane & 7;
#pragma unroll
            for (int mt = 0; mt < COUT / 16; ++mt)
                ldsm_x4_t(a[mt], sb + (16 * ks + rr + ((mat & 2) ? 8 : 0)) * LDY + 16 * mt + ((mat & 1) ? 8 : 0));
#pragma unroll
            for (int q = 0; q < PER; ++q) {
                if (wt + WPT * q >= T) break;
                // B = x (rows position, cols ci) at the tap's shifted slab rows
                uint32_t b0, b1;
                ldsm_x2_t(b0, b1, sb + boff[q] + 16 * ks * LDX);
                mma16816(acc[q], a[mtile[q]], b0, b1);
            }
        }
        __syncthreads();  // stage k & 1 is refilled by the next iteration's copies
    }
    asm volatile("cp.async.wait_all;" ::: "memory");
    const int gq = lane >> 2, tig = lane & 3;
#pragma unroll
    for (int q = 0; q < PER; ++q) {
        const int id = wt + WPT * q;
        if (id >= T) break;
        const int j = id / ((COUT / 16) * (CIN / 8)), rem = id - j * ((COUT / 16) * (CIN / 8));
        const int m0 = 16 * (rem / (CIN / 8)), n0 = 8 * (rem % (CIN / 8));
        float* w = dW + int64_t(g * TPG + j) * cout_real * CIN;  // rows past the real output channels are padding
        if (m0 + gq < cout_real) {
            atomicAdd(w + (m0 + gq) * CIN + n0 + 2 * tig, acc[q][0]);
            atomicAdd(w + (m0 + gq) * CIN + n0 + 2 * tig + 1, acc[q][1]);
        }
        if (m0 + gq + 8 < cout_real) {
            atomicAdd(w + (m0 + gq + 8) * CIN + n0 + 2 * tig, acc[q][2]);
            atomicAdd(w + (m0 + gq + 8) * CIN + n0 + 2 * tig + 1, acc[q][3]);
        }
    }
}

// ---- element-wise kernels ---------------------------------------------------------------

// masked output gradient (BF16, plain ld = C): m = dy * [y > 0] (relu) or dy
__global__ void k_grad_mask(TView dy, TView y, int relu, bf16* __restrict__ m, int C, int64_t nvox) {
    // one thread per (voxel, 4 channels): C, the views' ld and c0 are multiples of 4
    const int C4 = C / 4;
    const int64_t total = nvox * C4;
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < total; i += int64_t(gridDim.x) * blockDim.x) {
        const uint32_t v = uint32_t(i / C4);
        const int c = 4 * int(i - int64_t(v) * C4);
        const Vox q = vox_of(dy, v);
        const int64_t hv = hpos(dy, q.b, q.z, q.y, q.x);
        const float4 d = *reinterpret_cast<const float4*>(static_cast<const float*>(dy.p) + hv * dy.ld + dy.c0 + c);
        float val[4] = {d.x, d.y, d.z, d.w};
        if (relu) {
            const uint2 yy = *reinterpret_cast<const uint2*>(static_cast<const bf16*>(y.p) + hv * y.ld + y.c0 + c);
            const __nv_bfloat162 y01 = *reinterpret_cast<const __nv_bfloat162*>(&yy.x);
            const __nv_bfloat162 y23 = *reinterpret_cast<const __nv_bfloat162*>(&yy.y);
            if (!(__low2float(y01) > 0.f)) val[0] = 0.f;
            if (!(__high2float(y01) > 0.f)) val[1] = 0.f;
            if (!(__low2float(y23) > 0.f)) val[2] = 0.f;
            if (!(__high2float(y23) > 0.f)) val[3] = 0.f;
        }
        uint2 o;
        o.x = pack_bf16(val[0], val[1]);
        o.y = pack_bf16(val[2], val[3]);
        *reinterpret_cast<uint2*>(m + hv * C + c) = o;
    }
}

// db[c] += sum over every haloed position p of m[p][c] for c < count (m: C channels per position,
// C in {16, 32, 64}; its halo holds zeros, so the sum over all positions is the interior sum).
// Every thread sums one channel (blockDim and the grid stride are multiples of C) over a strided
// range, the block combines per channel in shared memory, and one atomic per channel and block
// adds to db.
__global__ void __launch_bounds__(256) k_bias_grad(const bf16* __restrict__ m, int64_t total, int C, int count,
                                                   float* __restrict__ db) {
    __shared__ float sh[64];
    if (threadIdx.x < 64) sh[threadIdx.x] = 0.f;
    __syncthreads();
    float s = 0.f;
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < total; i += int64_t(gridDim.x) * blockDim.x)
        s += __bfloat162float(m[i]);
    atomicAdd(&sh[threadIdx.x % C], s);
    __syncthreads();
    if (threadIdx.x < count) atomicAdd(db + threadIdx.x, sh[threadIdx.x]);
}

// 2x2x2 average pooling: out (extents of the coarse grid) from in (twice as fine); one thread
// per (coarse voxel, 8 channels): eight 16-byte loads, one 16-byte store (C, ld and c0 are
// multiples of 8).  Index arithmetic in 32 bits: every grid holds fewer than 2^31 positions.
__global__ void k_pool(TView in, TView out, int C) {
    const int C8 = C / 8;
    const int64_t total = int64_t(out.B) * out.D * out.H * out.W * C8;
    const int32_t fy = in.W + 2, fz = (in.H + 2) * fy;
    const bf16* __restrict__ ip = static_cast<const bf16*>(in.p);
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < total; i += int64_t(gridDim.x) * blockDim.x) {
        const uint32_t v = uint32_t(i / C8);
        const int c = 8 * int(i - int64_t(v) * C8);
        const Vox q = vox_of(out, v);
        const int32_t f = hpos(in, q.b, 2 * q.z, 2 * q.y, 2 * q.x);
        float s[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            const int32_t p = f + (k >> 2) * fz + ((k >> 1) & 1) * fy + (k & 1);
            const uint4 u = *reinterpret_cast<const uint4*>(ip + int64_t(p) * in.ld + in.c0 + c);
            const uint32_t w[4] = {u.x, u.y, u.z, u.w};
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const __nv_bfloat162 h = *reinterpret_cast<const __nv_bfloat162*>(&w[j]);
                s[2 * j] += __low2float(h);
                s[2 * j + 1] += __high2float(h);
            }
        }
        uint4 o;
        o.x = pack_bf16(0.125f * s[0], 0.125f * s[1]);
        o.y = pack_bf16(0.125f * s[2], 0.125f * s[3]);
        o.z = pack_bf16(0.125f * s[4], 0.125f * s[5]);
        o.w = pack_bf16(0.125f * s[6], 0.125f * s[7]);
        *reinterpret_cast<uint4*>(static_cast<bf16*>(out.p) + int64_t(hpos(out, q.b, q.z, q.y, q.x)) * out.ld + out.c0 + c) = o;
    }
}

// pooling gradient: din[fine] += dout[coarse] / 8 (FP32 gradients); one thread per (coarse
// voxel, 4 channels), one float4 read and eight float4 read-modify-writes
__global__ void k_pool_grad(TView dout, TView din, int C) {
    const int C4 = C / 4;
    const int64_t total = int64_t(dout.B) * dout.D * dout.H * dout.W * C4;
    const int32_t fy = din.W + 2, fz = (din.H + 2) * fy;
    float* __restrict__ dp = static_cast<float*>(din.p);
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < total; i += int64_t(gridDim.x) * blockDim.x) {
        const uint32_t v = uint32_t(i / C4);
        const int c = 4 * int(i - int64_t(v) * C4);
        const Vox q = vox_of(dout, v);
        const float4 g = *reinterpret_cast<const float4*>(static_cast<const float*>(dout.p) +
                                                          int64_t(hpos(dout, q.b, q.z, q.y, q.x)) * dout.ld + dout.c0 + c);
        const int32_t f = hpos(din, q.b, 2 * q.z, 2 * q.y, 2 * q.x);
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            const int32_t p = f + (k >> 2) * fz + ((k >> 1) & 1) * fy + (k & 1);
            float4* o = reinterpret_cast<float4*>(dp + int64_t(p) * din.ld + din.c0 + c);
            float4 a = *o;
            a.x += 0.125f * g.x; a.y += 0.125f * g.y; a.z += 0.125f * g.z; a.w += 0.125f * g.w;
            *o = a;
        }
    }
}

// nearest upsampling: out[fine] = in[coarse]; one thread per (coarse voxel, 8 channels), one
// 16-byte load and eight 16-byte stores
__global__ void k_upsample(TView in, TView out, int C) {
    const int C8 = C / 8;
    const int64_t total = int64_t(in.B) * in.D * in.H * in.W * C8;
    const int32_t fy = out.W + 2, fz = (out.H + 2) * fy;
    bf16* __restrict__ op = static_cast<bf16*>(out.p);
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < total; i += int64_t(gridDim.x) * blockDim.x) {
        const uint32_t v = uint32_t(i / C8);
        const int c = 8 * int(i - int64_t(v) * C8);
        const Vox q = vox_of(in, v);
        const uint4 u = *reinterpret_cast<const uint4*>(static_cast<const bf16*>(in.p) +
                                                        int64_t(hpos(in, q.b, q.z, q.y, q.x)) * in.ld + in.c0 + c);
        const int32_t f = hpos(out, q.b, 2 * q.z, 2 * q.y, 2 * q.x);
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            const int32_t p = f + (k >> 2) * fz + ((k >> 1) & 1) * fy + (k & 1);
            *reinterpret_cast<uint4*>(op + int64_t(p) * out.ld + out.c0 + c) = u;
        }
    }
}

// upsampling gradient: din[coarse] = sum of the 8 fine dout; one thread per (coarse voxel,
// 4 channels), eight float4 loads summed in the fine voxels' order
__global__ void k_upsample_grad(TView dout, TView din, int C) {
    const int C4 = C / 4;
    const int64_t total = int64_t(din.B) * din.D * din.H * din.W * C4;
    const int32_t fy = dout.W + 2, fz = (dout.H + 2) * fy;
    const float* __restrict__ gp = static_cast<const float*>(dout.p);
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < total; i += int64_t(gridDim.x) * blockDim.x) {
        const uint32_t v = uint32_t(i / C4);
        const int c = 4 * int(i - int64_t(v) * C4);
        const Vox q = vox_of(din, v);
        const int32_t f = hpos(dout, q.b, 2 * q.z, 2 * q.y, 2 * q.x);
        float4 s = make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            const int32_t p = f + (k >> 2) * fz + ((k >> 1) & 1) * fy + (k & 1);
            const float4 a = *reinterpret_cast<const float4*>(gp + int64_t(p) * dout.ld + dout.c0 + c);
            s.x += a.x; s.y += a.y; s.z += a.z; s.w += a.w;
        }
        *reinterpret_cast<float4*>(static_cast<float*>(din.p) + int64_t(hpos(din, q.b, q.z, q.y, q.x)) * din.ld + din.c0 + c) = s;
    }
}

// network input: plain FP32 [B][n0][n1][n2][8] nodes -> haloed BF16 (16 channels, 8..15 zero);
// one thread per node: two float4 loads, one 16-byte store
__global__ void k_pack_input(const float* __restrict__ src, int n0, int n1, int n2, TView in) {
    const int64_t nv = int64_t(in.B) * n0 * n1 * n2;
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < nv; i += int64_t(gridDim.x) * blockDim.x) {
        uint32_t v = uint32_t(i);
        const int x = int(v % uint32_t(n2));
        v /= uint32_t(n2);
        const int y = int(v % uint32_t(n1));
        v /= uint32_t(n1);
        const int z = int(v % uint32_t(n0));
        const int b = int(v / uint32_t(n0));
        const float4 a = reinterpret_cast<const float4*>(src)[2 * i];
        const float4 c = reinterpret_cast<const float4*>(src)[2 * i + 1];
        uint4 o;
        o.x = pack_bf16(a.x, a.y);
        o.y = pack_bf16(a.z, a.w);
        o.z = pack_bf16(c.x, c.y);
        o.w = pack_bf16(c.z, c.w);
        *reinterpret_cast<uint4*>(static_cast<bf16*>(in.p) + int64_t(hpos(in, b, z, y, x)) * in.ld) = o;
    }
}

// network output: haloed FP32 (ld 16, 9 channels) -> plain FP32 [B][n0][n1][n2][9]
__global__ void k_unpack_output(TView out, int n0, int n1, int n2, float* __restrict__ dst) {
    const int64_t nv = int64_t(out.B) * n0 * n1 * n2;
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < nv * 9; i += int64_t(gridDim.x) * blockDim.x) {
        uint32_t v = uint32_t(i / 9);
        const int c = int(i - int64_t(v) * 9);
        const int x = int(v % uint32_t(n2));
        v /= uint32_t(n2);
        const int y = int(v % uint32_t(n1));
        v /= uint32_t(n1);
        const int z = int(v % uint32_t(n0));
        const int b = int(v / uint32_t(n0));
        dst[i] = static_cast<const float*>(out.p)[int64_t(hpos(out, b, z, y, x)) * out.ld + c];
    }
}

// mean squared error over the node region and its gradient (zero on padding voxels); one
// thread per voxel of the padded grid: the 16-channel output row in four float4 loads, the
// BF16 gradient row in two 16-byte stores
__global__ void k_loss(TView out, const float* __restrict__ tgt, int n0, int n1, int n2, TView dout,
                       double* __restrict__ loss) {
    const int64_t nv = int64_t(out.B) * out.D * out.H * out.W;
    const double inv = 1.0 / (double(out.B) * n0 * n1 * n2 * 9);
    const float g2 = float(2.0 * inv);
    double local = 0.0;
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < nv; i += int64_t(gridDim.x) * blockDim.x) {
        const Vox q = vox_of(out, uint32_t(i));
        const int32_t hv = hpos(out, q.b, q.z, q.y, q.x);
        float gval[16];
#pragma unroll
        for (int c = 0; c < 16; ++c) gval[c] = 0.f;
        if (q.z < n0 && q.y < n1 && q.x < n2) {
            const float4* orow = reinterpret_cast<const float4*>(static_cast<const float*>(out.p) + int64_t(hv) * out.ld);
            float o[12];
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                const float4 a = orow[k];
                o[4 * k] = a.x; o[4 * k + 1] = a.y; o[4 * k + 2] = a.z; o[4 * k + 3] = a.w;
            }
            const float* t = tgt + ((((int64_t(q.b) * n0 + q.z) * n1 + q.y) * n2 + q.x) * 9);
#pragma unroll
            for (int c = 0; c < 9; ++c) {
                const float d = o[c] - t[c];
                local += double(d) * d;
                gval[c] = g2 * d;
            }
        }
        uint4 lo, hi;
        lo.x = pack_bf16(gval[0], gval[1]); lo.y = pack_bf16(gval[2], gval[3]);
        lo.z = pack_bf16(gval[4], gval[5]); lo.w = pack_bf16(gval[6], gval[7]);
        hi.x = pack_bf16(gval[8], gval[9]); hi.y = pack_bf16(gval[10], gval[11]);
        hi.z = pack_bf16(gval[12], gval[13]); hi.w = pack_bf16(gval[14], gval[15]);
        uint4* drow = reinterpret_cast<uint4*>(static_cast<bf16*>(dout.p) + int64_t(hv) * dout.ld);
        drow[0] = lo;
        drow[1] = hi;
    }
    for (int o = 16; o > 0; o >>= 1) local += __shfl_xor_sync(0xffffffffu, local, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(loss, local * inv);
}

// Adam (Kingma & Ba) on the FP32 parameters
__global__ void k_adam(int64_t n, float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                       float* __restrict__ v, float lr, float b1, float b2, float eps, float c1, float c2) {
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.f - b1) * gi;
        const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    }
}

// BF16 copies of a layer's weights: forward [t][co][ci] and data-gradient [t'][ci][co]
// with t' = taps - 1 - t (flipped kernel, transposed channels)
__global__ void k_pack_weights(const float* __restrict__ w, int taps, int cout, int coutp, int cin,
                               bf16* __restrict__ wf, bf16* __restrict__ wb, int cinp_b) {
    const int64_t n = int64_t(taps) * coutp * cin;
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
        const int ci = int(i % cin);
        const int co = int((i / cin) % coutp);
        const int t = int(i / (int64_t(cin) * coutp));
        const float val = co < cout ? w[(int64_t(t) * cout + co) * cin + ci] : 0.f;
        wf[i] = __float2bfloat16(val);
        if (wb && co < cinp_b) wb[(int64_t(taps - 1 - t) * cin + ci) * cinp_b + co] = __float2bfloat16(val);
    }
}

// trilinear interpolation on a box node grid (nodes z fastest) at fractional index (fx, fy, fz)
__device__ __forceinline__ void trilinear_setup(double f, int s, int& i0, double& u) {
    i0 = min(int(floor(f)), s > 1 ? s - 2 : 0);
    u = f - i0;
}

// trilinear resampling between two node grids spanning the same box (nodes z fastest)
__global__ void k_box_resample(int s0, int s1, int s2, int d0, int d1, int d2, int C, const double* __restrict__ src,
                               double* __restrict__ dst) {
    const int64_t n = int64_t(d0) * d1 * d2;
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
        const int k = int(i % d2), j = int((i / d2) % d1), l = int(i / (int64_t(d2) * d1));
        int x0, y0, z0;
        double ux, uy, uz;
        trilinear_setup(d0 > 1 ? double(l) * (s0 - 1) / (d0 - 1) : 0.0, s0, x0, ux);
        trilinear_setup(d1 > 1 ? double(j) * (s1 - 1) / (d1 - 1) : 0.0, s1, y0, uy);
        trilinear_setup(d2 > 1 ? double(k) * (s2 - 1) / (d2 - 1) : 0.0, s2, z0, uz);
        for (int c = 0; c < C; ++c) {
            double s = 0.0;
            for (int q = 0; q < 8; ++q) {
                const int xx = min(x0 + (q >> 2), s0 - 1), yy = min(y0 + ((q >> 1) & 1), s1 - 1), zz = min(z0 + (q & 1), s2 - 1);
                const double w = ((q >> 2) ? ux : 1.0 - ux) * (((q >> 1) & 1) ? uy : 1.0 - uy) * ((q & 1) ? uz : 1.0 - uz);
                s += w * src[((int64_t(xx) * s1 + yy) * s2 + zz) * C + c];
            }
            dst[i * C + c] = s;
        }
    }
}

// network features of a box design on the network's node grid, from the nodal density of a
// (possibly finer) box node grid: 0 density (trilinear), 1 loaded face x = max, 2 clamped face
// x = 0, 3..5 normalised node coordinates, 6 density cubed (the SIMP stiffness scale), 7 zero
__global__ void k_features(int s0, int s1, int s2, const double* __restrict__ z, int n0, int n1, int n2,
                           float* __restrict__ feat) {
    const int64_t n = int64_t(n0) * n1 * n2;
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
        const int k = int(i % n2), j = int((i / n2) % n1), l = int(i / (int64_t(n2) * n1));
        int x0, y0, z0;
        double ux, uy, uz;
        trilinear_setup(n0 > 1 ? double(l) * (s0 - 1) / (n0 - 1) : 0.0, s0, x0, ux);
        trilinear_setup(n1 > 1 ? double(j) * (s1 - 1) / (n1 - 1) : 0.0, s1, y0, uy);
        trilinear_setup(n2 > 1 ? double(k) * (s2 - 1) / (n2 - 1) : 0.0, s2, z0, uz);
        double d = 0.0;
        for (int q = 0; q < 8; ++q) {
            const int xx = min(x0 + (q >> 2), s0 - 1), yy = min(y0 + ((q >> 1) & 1), s1 - 1), zz = min(z0 + (q & 1), s2 - 1);
            d += ((q >> 2) ? ux : 1.0 - ux) * (((q >> 1) & 1) ? uy : 1.0 - uy) * ((q & 1) ? uz : 1.0 - uz) *
                 z[(int64_t(xx) * s1 + yy) * s2 + zz];
        }
        float* f = feat + 8 * i;
        f[0] = float(d);
        f[1] = l == n0 - 1 ? 1.f : 0.f;
        f[2] = l == 0 ? 1.f : 0.f;
        f[3] = n0 > 1 ? float(l) / float(n0 - 1) : 0.f;
        f[4] = n1 > 1 ? float(j) / float(n1 - 1) : 0.f;
        f[5] = n2 > 1 ? float(k) / float(n2 - 1) : 0.f;
        f[6] = float(d * d * d);
        f[7] = 0.f;
    }
}

// subspace columns on a (possibly finer) box node grid from the network output: column d
// (d = load direction) at node p, component c = trilinear interpolation of output channel 3d + c
__global__ void k_subspace(int n0, int n1, int n2, const float* __restrict__ out9, int d0, int d1, int d2,
                           double* __restrict__ W) {
    const int64_t n = int64_t(d0) * d1 * d2;
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
        const int k = int(i % d2), j = int((i / d2) % d1), l = int(i / (int64_t(d2) * d1));
        int x0, y0, z0;
        double ux, uy, uz;
        trilinear_setup(d0 > 1 ? double(l) * (n0 - 1) / (d0 - 1) : 0.0, n0, x0, ux);
        trilinear_setup(d1 > 1 ? double(j) * (n1 - 1) / (d1 - 1) : 0.0, n1, y0, uy);
        trilinear_setup(d2 > 1 ? double(k) * (n2 - 1) / (d2 - 1) : 0.0, n2, z0, uz);
        double acc[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
        for (int q = 0; q < 8; ++q) {
            const int xx = min(x0 + (q >> 2), n0 - 1), yy = min(y0 + ((q >> 1) & 1), n1 - 1), zz = min(z0 + (q & 1), n2 - 1);
            const double w = ((q >> 2) ? ux : 1.0 - ux) * (((q >> 1) & 1) ? uy : 1.0 - uy) * ((q & 1) ? uz : 1.0 - uz);
            const float* o = out9 + ((int64_t(xx) * n1 + yy) * n2 + zz) * 9;
            for (int c = 0; c < 9; ++c) acc[c] += w * double(o[c]);
        }
        for (int dcol = 0; dcol < 3; ++dcol)
            for (int c = 0; c < 3; ++c) W[dcol * 3 * n + 3 * i + c] = acc[3 * dcol + c];
    }
}

// one 7-point averaging pass over a box node grid (C values per node): each node becomes the
// mean of itself and its face neighbours inside the grid
__global__ void k_box_smooth(int n0, int n1, int n2, int C, const float* __restrict__ in, float* __restrict__ out) {
    const int64_t n = int64_t(n0) * n1 * n2;
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n * C; i += int64_t(gridDim.x) * blockDim.x) {
        const int64_t v = i / C;
        const int k = int(v % n2), j = int((v / n2) % n1), l = int(v / (int64_t(n2) * n1));
        float s = in[i];
        int cnt = 1;
        const int64_t sx = int64_t(n1) * n2 * C, sy = int64_t(n2) * C;
        if (l > 0) { s += in[i - sx]; ++cnt; }
        if (l < n0 - 1) { s += in[i + sx]; ++cnt; }
        if (j > 0) { s += in[i - sy]; ++cnt; }
        if (j < n1 - 1) { s += in[i + sy]; ++cnt; }
        if (k > 0) { s += in[i - C]; ++cnt; }
        if (k < n2 - 1) { s += in[i + C]; ++cnt; }
        out[i] = s / float(cnt);
    }
}

int blocks_for(int64_t n, int threads, int64_t cap = 148 * 32) {
    int64_t b = (n + threads - 1) / threads;
    if (b < 1) b = 1;
    return int(b < cap ? b : cap);
}

// ---- the network ------------------------------------------------------------------------

struct Layer {
    int cin, cout, taps, relu;
    int64_t w_off, b_off;     // offsets in the FP32 parameter vector
    bf16* wf = nullptr;       // [taps][coutp][cin]
    bf16* wb = nullptr;       // [taps][cin][coutp_b] (data gradient)
    int coutp() const { return (cout + 7) / 8 * 8; }
};

}  // namespace

struct plato_unet {
    cudaStream_t stream = nullptr;
    int n[3] = {0, 0, 0};        // node grid
    int g0[3] = {0, 0, 0};       // padded level-0 grid (multiples of 4)
    int max_batch = 0;
    std::vector<Layer> layers;   // e0a e0b e1a e1b e2a e2b d1a d1b d0a d0b head
    int64_t nparams = 0;
    float *params = nullptr, *grads = nullptr, *adam_m = nullptr, *adam_v = nullptr;
    // activations (BF16, haloed) and gradients (FP32, haloed)
    bf16 *in = nullptr, *x0a = nullptr, *cat0 = nullptr, *p1 = nullptr, *x1a = nullptr, *cat1 = nullptr,
         *p2 = nullptr, *x2a = nullptr, *x2b = nullptr, *x1c = nullptr, *x1d = nullptr, *x0c = nullptr, *x0d = nullptr;
    float* out = nullptr;
    float *dx0a = nullptr, *dcat0 = nullptr, *dp1 = nullptr, *dx1a = nullptr, *dcat1 = nullptr, *dp2 = nullptr,
          *dx2a = nullptr, *dx2b = nullptr, *dx1c = nullptr, *dx1d = nullptr, *dx0c = nullptr, *dx0d = nullptr;
    int conv_kind = PLATO_UNET_CONV_TCGEN05;
    int* conv_err = nullptr;     // raised by a tcgen05 convolution whose bounded wait ran out
    bf16* mbuf = nullptr;        // masked output gradient (BF16), also the head's gradient
    double* loss_d = nullptr;
    std::vector<void*> allocs;
};

namespace {

int64_t halo_elems(const int* g, int B, int C) { return int64_t(B) * (g[0] + 2) * (g[1] + 2) * (g[2] + 2) * C; }

TView tv(void* p, int ld, int c0, int B, const int* g) { return TView{p, ld, c0, B, g[0], g[1], g[2]}; }

template <typename T>
int alloc(plato_unet* u, T** p, int64_t count) {
    UCUDA(cudaMalloc(reinterpret_cast<void**>(p), sizeof(T) * size_t(count > 0 ? count : 1)));
    u->allocs.push_back(*p);
    UCUDA(cudaMemset(*p, 0, sizeof(T) * size_t(count > 0 ? count : 1)));
    return PLATO_OK;
}

// The convolution kernel family of a network: tcgen05 (default) or the warp-level mma.sync form.
struct ConvPath {
    int kind;  // PLATO_UNET_CONV_TCGEN05 or PLATO_UNET_CONV_MMA_SYNC
    int* err;  // device flag raised by a tcgen05 CTA whose bounded wait ran out
};

int sm_count() {
    static const int n = [] {
        int dev = 0, v = 148;
        if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
            v = 148;
        return v;
    }();
    return n;
}

// Shared memory and pipeline of a k_conv_tc launch with slab row stride `rows`: every tap's
// weights stay resident when they fit beside two slab buffers (else each buffer carries its
// slab's 9 taps); then the buffer count (2 to 4) that keeps the most slab copies in flight per
// SM, resident CTAs x (buffers - 1), fewer buffers on a tie.  The dynamic shared memory is
// raised so that no more CTAs fit on an SM than its 512 TMEM columns hold (a CTA beyond them
// would wait in tcgen05.alloc for a persistent CTA to end).  False when no form fits.
template <int CIN, int COUTP, int TAPS>
bool tc_plan(int rows, TcGeom& g, uint32_t& smem, int& ctas_per_sm) {
    constexpr int TPD = TAPS == 27 ? 9 : 1;
    constexpr uint32_t BTAP = uint32_t(COUTP) * CIN * 2;
    constexpr uint32_t kMaxDyn = 227u * 1024u - 1280u;  // the opt-in limit less the static mbarriers and bias
    constexpr uint32_t kSmPerSm = 228u * 1024u, kPerCtaExtra = 1024u + 1280u;  // reserved + static per CTA
    constexpr int tmem_ctas = 512 / (2 * tc_tmem_cols<COUTP>());
    auto r128 = [](uint32_t v) { return (v + 127u) & ~127u; };
    const uint32_t a = r128(uint32_t(rows) * CIN * 2), wall = r128(uint32_t(TAPS) * BTAP);
    const bool wres = wall + 2u * a <= kMaxDyn;
    const uint32_t wb = wres ? wall : 0u, buf = wres ? a : r128(a + uint32_t(TPD) * BTAP);
    const uint32_t guard = (227u * 1024u) / uint32_t(tmem_ctas) + 1024u;
    int best = 0;
    for (int nb = 2; nb <= 4; ++nb) {
        const uint32_t need = std::max(wb + uint32_t(nb) * buf, guard);
        if (need > kMaxDyn) break;
        const int occ = std::min<int>(tmem_ctas, int(kSmPerSm / (need + kPerCtaExtra)));
        const int lag = nb - 1;  // measured alike with lag nb - 2 (one iteration of MMA slack)
        const int score = occ * lag;
        if (score > best) {
            best = score;
            g.nbuf = nb;
            g.lag = lag;
            smem = need;
            ctas_per_sm = occ;
        }
    }
    if (best == 0) return false;
    g.rows = rows;
    g.wres = wres ? 1 : 0;
    g.w_bytes = wb;
    g.buf_bytes = buf;
    return true;
}

// launch helpers (dispatch on the layer's channel counts)
template <int CIN, int COUT, int TAPS, bool RELU, bool F32, bool ACC>
int conv_launch(cudaStream_t s, const ConvPath& P, TView in, const bf16* w, const float* b, TView out, int64_t nvox) {
    if (nvox <= 0) return PLATO_OK;
    if (in.B != out.B || in.D != out.D || in.H != out.H || in.W != out.W)
        return fail(PLATO_BAD_INPUT, "convolution input and output grids differ");
    if (P.kind == PLATO_UNET_CONV_TCGEN05) {
        constexpr int COUTP = (COUT + 15) / 16 * 16;
        const int64_t sy = in.W + 2, sz = int64_t(in.H + 2) * sy;
        const int64_t ptotal = int64_t(in.B) * (in.D + 2) * sz;
        const int nrows = kTcRows + (TAPS == 27 ? 2 * int(sy + 1) : 0);
        TcGeom g{};
        uint32_t smem = 0;
        int ctas_per_sm = 0;
        // positions index in 32 bits; a slab too long for shared memory (a grid row of more than
        // about 140 voxels on the widest layers) takes the mma.sync kernel
        if (ptotal < (int64_t(1) << 31) && tc_plan<CIN, COUTP, TAPS>(tc_row_stride(nrows, CIN / 8), g, smem, ctas_per_sm)) {
            g.pfirst = int32_t(sz + sy + 1);
            g.plast = int32_t(halo_index(in, nvox - 1));
            g.ptotal = int32_t(ptotal);
            g.ntiles = (g.plast - g.pfirst) / kTcRows + 1;
            auto kernel = k_conv_tc<CIN, COUT, TAPS, RELU, F32, ACC>;
            UCUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
            const int grid = int(std::min<int64_t>(g.ntiles, int64_t(sm_count()) * ctas_per_sm));
            kernel<<<grid, 128, smem, s>>>(in, w, b, out, g, P.err);
            ULAUNCH();
            return PLATO_OK;
        }
    }
    const int64_t per = kConvWarps * 16 * kMT;
    k_conv<CIN, COUT, TAPS, RELU, F32, ACC><<<int((nvox + per - 1) / per), kConvWarps * 32, 0, s>>>(in, w, b, out, nvox);
    ULAUNCH();
    return PLATO_OK;
}

int conv_forward(cudaStream_t s, const ConvPath& P, const Layer& L, TView in, TView out, const float* bias,
                 int64_t nvox) {
    const int c = L.cin, o = L.cout;
    if (L.taps == 1) return conv_launch<16, 9, 1, false, true, false>(s, P, in, L.wf, bias, out, nvox);
#define FWD(CI, CO) \
    if (c == CI && o == CO) return conv_launch<CI, CO, 27, true, false, false>(s, P, in, L.wf, bias, out, nvox);
    FWD(16, 16) FWD(16, 32) FWD(32, 32) FWD(32, 64) FWD(64, 64) FWD(96, 32) FWD(48, 16)
#undef FWD
    return fail(PLATO_NOT_SUPPORTED, "no forward convolution for these channel counts");
}

// data gradient into an FP32 tensor (write, or accumulate)
int conv_data_grad(cudaStream_t s, const ConvPath& P, const Layer& L, TView dy, TView dx, int64_t nvox,
                   bool accumulate) {
    const int c = L.cout, o = L.cin;  // roles swap
    if (L.taps == 1) {
        if (accumulate) return conv_launch<16, 16, 1, false, true, true>(s, P, dy, L.wb, nullptr, dx, nvox);
        return conv_launch<16, 16, 1, false, true, false>(s, P, dy, L.wb, nullptr, dx, nvox);
    }
#define BWD(CI, CO)                                                                                          \
    if (c == CI && o == CO) {                                                                                \
        if (accumulate) return conv_launch<CI, CO, 27, false, true, true>(s, P, dy, L.wb, nullptr, dx, nvox); \
        return conv_launch<CI, CO, 27, false, true, false>(s, P, dy, L.wb, nullptr, dx, nvox);               \
    }
    BWD(16, 16) BWD(32, 16) BWD(32, 32) BWD(64, 32) BWD(64, 64) BWD(32, 96) BWD(16, 48)
#undef BWD
    return fail(PLATO_NOT_SUPPORTED, "no data-gradient convolution for these channel counts");
}

template <int CIN, int COUT, int TAPS>
int wgrad_launch(cudaStream_t s, TView x, TView dy, float* dW, int cout_real, int64_t nvox) {
    if (nvox <= 0) return PLATO_OK;
    if (x.B != dy.B || x.D != dy.D || x.H != dy.H || x.W != dy.W)
        return fail(PLATO_BAD_INPUT, "weight gradient: input and output grids differ");
    constexpr int G = wg_groups<CIN, COUT, TAPS>();
    constexpr int NSL = (TAPS == 27 && G == 1) ? 3 : 1;
    const int64_t sy = x.W + 2, sz = int64_t(x.H + 2) * sy;
    const int64_t ptotal = int64_t(x.B) * (x.D + 2) * sz;
    if (ptotal >= (int64_t(1) << 31)) return fail(PLATO_NOT_SUPPORTED, "weight gradient: grid above 2^31 positions");
    const int srows = kWgRows + 2 * wg_halfwidth<TAPS, G>(int(sy));
    const int rows_pad = srows;
    const uint32_t stage_elems = uint32_t(kWgRows * (COUT + 8) + NSL * rows_pad * (CIN + 8));
    const uint32_t smem = 2u * stage_elems * 2u;
    if (smem > 227u * 1024u) return fail(PLATO_NOT_SUPPORTED, "weight gradient: grid rows too long for shared memory");
    auto kernel = k_conv_wgrad<CIN, COUT, TAPS, G>;
    UCUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
    int occ = 0;
    UCUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kernel, 128, smem));
    const int32_t pfirst = int32_t(sz + sy + 1), plast = int32_t(halo_index(x, nvox - 1));
    const int32_t ntiles = (plast - pfirst) / kWgRows + 1;
    const int gx = int(std::max<int64_t>(1, std::min<int64_t>(ntiles, int64_t(sm_count()) * std::max(occ, 1) / G)));
    kernel<<<dim3(unsigned(gx), unsigned(G)), 128, smem, s>>>(x, dy, dW, cout_real, pfirst, plast, int32_t(ptotal), ntiles,
                                                               rows_pad, stage_elems);
    ULAUNCH();
    return PLATO_OK;
}

int conv_weight_grad(cudaStream_t s, const Layer& L, TView x, TView dy, float* dW, int64_t nvox) {
    const int c = L.cin, o = L.coutp() < 16 ? 16 : L.coutp();
    if (L.taps == 1) return wgrad_launch<16, 16, 1>(s, x, dy, dW, L.cout, nvox);
#define WG(CI, CO) \
    if (c == CI && o == CO) return wgrad_launch<CI, CO, 27>(s, x, dy, dW, L.cout, nvox);
    WG(16, 16) WG(16, 32) WG(32, 32) WG(32, 64) WG(64, 64) WG(96, 32) WG(48, 16)
#undef WG
    return fail(PLATO_NOT_SUPPORTED, "no weight-gradient kernel for these channel counts");
}

#define URC(expr)                    \
    do {                             \
        int _rc = (expr);            \
        if (_rc) return _rc;         \
    } while (0)

int pack_all_weights(plato_unet* u) {
    for (Layer& L : u->layers) {
        const int64_t n = int64_t(L.taps) * L.coutp() * L.cin;
        const int cinp_b = L.taps == 1 ? 16 : L.coutp();
        k_pack_weights<<<blocks_for(n, 256), 256, 0, u->stream>>>(u->params + L.w_off, L.taps, L.cout, L.coutp(), L.cin,
                                                                 L.wf, L.wb, cinp_b);
        ULAUNCH();
    }
    return PLATO_OK;
}

int forward(plato_unet* u, int B, const float* input) {
    cudaStream_t s = u->stream;
    const int* G0 = u->g0;
    const int G1[3] = {G0[0] / 2, G0[1] / 2, G0[2] / 2};
    const int G2[3] = {G1[0] / 2, G1[1] / 2, G1[2] / 2};
    const int64_t n0 = int64_t(B) * G0[0] * G0[1] * G0[2], n1 = int64_t(B) * G1[0] * G1[1] * G1[2],
                  n2 = int64_t(B) * G2[0] * G2[1] * G2[2];
    const std::vector<Layer>& L = u->layers;
    const ConvPath P{u->conv_kind, u->conv_err};
    auto bias = [&](int k) { return u->params + L[k].b_off; };
    const int64_t nn = int64_t(B) * u->n[0] * u->n[1] * u->n[2];
    k_pack_input<<<blocks_for(nn, 256), 256, 0, s>>>(input, u->n[0], u->n[1], u->n[2], tv(u->in, 16, 0, B, G0));
    ULAUNCH();
    URC(conv_forward(s, P, L[0], tv(u->in, 16, 0, B, G0), tv(u->x0a, 16, 0, B, G0), bias(0), n0));
    URC(conv_forward(s, P, L[1], tv(u->x0a, 16, 0, B, G0), tv(u->cat0, 48, 32, B, G0), bias(1), n0));
    k_pool<<<blocks_for(n1 * 2, 256), 256, 0, s>>>(tv(u->cat0, 48, 32, B, G0), tv(u->p1, 16, 0, B, G1), 16);
    ULAUNCH();
    URC(conv_forward(s, P, L[2], tv(u->p1, 16, 0, B, G1), tv(u->x1a, 32, 0, B, G1), bias(2), n1));
    URC(conv_forward(s, P, L[3], tv(u->x1a, 32, 0, B, G1), tv(u->cat1, 96, 64, B, G1), bias(3), n1));
    k_pool<<<blocks_for(n2 * 4, 256), 256, 0, s>>>(tv(u->cat1, 96, 64, B, G1), tv(u->p2, 32, 0, B, G2), 32);
    ULAUNCH();
    URC(conv_forward(s, P, L[4], tv(u->p2, 32, 0, B, G2), tv(u->x2a, 64, 0, B, G2), bias(4), n2));
    URC(conv_forward(s, P, L[5], tv(u->x2a, 64, 0, B, G2), tv(u->x2b, 64, 0, B, G2), bias(5), n2));
    k_upsample<<<blocks_for(n2 * 8, 256), 256, 0, s>>>(tv(u->x2b, 64, 0, B, G2), tv(u->cat1, 96, 0, B, G1), 64);
    ULAUNCH();
    URC(conv_forward(s, P, L[6], tv(u->cat1, 96, 0, B, G1), tv(u->x1c, 32, 0, B, G1), bias(6), n1));
    URC(conv_forward(s, P, L[7], tv(u->x1c, 32, 0, B, G1), tv(u->x1d, 32, 0, B, G1), bias(7), n1));
    k_upsample<<<blocks_for(n1 * 4, 256), 256, 0, s>>>(tv(u->x1d, 32, 0, B, G1), tv(u->cat0, 48, 0, B, G0), 32);
    ULAUNCH();
    URC(conv_forward(s, P, L[8], tv(u->cat0, 48, 0, B, G0), tv(u->x0c, 16, 0, B, G0), bias(8), n0));
    URC(conv_forward(s, P, L[9], tv(u->x0c, 16, 0, B, G0), tv(u->x0d, 16, 0, B, G0), bias(9), n0));
    URC(conv_forward(s, P, L[10], tv(u->x0d, 16, 0, B, G0), tv(u->out, 16, 0, B, G0), bias(10), n0));
    return PLATO_OK;
}

// one layer's backward: dY (FP32 slice) masked by its output -> weight and bias gradients,
// and (write_dx) the data gradient into dx (write, or accumulate)
int layer_backward(plato_unet* u, int k, TView dy, TView y, TView x, TView dx, bool write_dx, bool accumulate,
                   int64_t nvox) {
    cudaStream_t s = u->stream;
    const Layer& L = u->layers[k];
    const ConvPath P{u->conv_kind, u->conv_err};
    const int C = L.coutp() < 16 ? 16 : L.coutp();
    const int gdims[3] = {y.D, y.H, y.W};
    TView m = tv(u->mbuf, C, 0, y.B, gdims);
    if (k != int(u->layers.size()) - 1) {  // the head's masked gradient is written by the loss
        // mbuf is reused with other grids and widths: clear it so its halo reads as zero
        UCUDA(cudaMemsetAsync(u->mbuf, 0, sizeof(bf16) * size_t(halo_elems(gdims, y.B, C)), s));
        k_grad_mask<<<blocks_for(nvox * L.cout, 256), 256, 0, s>>>(dy, y, L.relu, u->mbuf, C, nvox);
        ULAUNCH();
    }
    URC(conv_weight_grad(s, L, x, m, u->grads + L.w_off, nvox));
    const int64_t mtotal = halo_elems(gdims, y.B, C);
    k_bias_grad<<<blocks_for(mtotal, 256, 148 * 8), 256, 0, s>>>(u->mbuf, mtotal, C, L.cout, u->grads + L.b_off);
    ULAUNCH();
    if (write_dx) URC(conv_data_grad(s, P, L, m, dx, nvox, accumulate));
    return PLATO_OK;
}

int backward(plato_unet* u, int B) {
    cudaStream_t s = u->stream;
    const int* G0 = u->g0;
    const int G1[3] = {G0[0] / 2, G0[1] / 2, G0[2] / 2};
    const int G2[3] = {G1[0] / 2, G1[1] / 2, G1[2] / 2};
    const int64_t n0 = int64_t(B) * G0[0] * G0[1] * G0[2], n1 = int64_t(B) * G1[0] * G1[1] * G1[2],
                  n2 = int64_t(B) * G2[0] * G2[1] * G2[2];
    TView none{nullptr, 0, 0, B, 1, 1, 1};
    UCUDA(cudaMemsetAsync(u->grads, 0, sizeof(float) * size_t(u->nparams), s));
    // head (its masked gradient, BF16, is in mbuf from the loss)
    URC(layer_backward(u, 10, none, tv(u->out, 16, 0, B, G0), tv(u->x0d, 16, 0, B, G0), tv(u->dx0d, 16, 0, B, G0),
                       true, false, n0));
    URC(layer_backward(u, 9, tv(u->dx0d, 16, 0, B, G0), tv(u->x0d, 16, 0, B, G0), tv(u->x0c, 16, 0, B, G0),
                       tv(u->dx0c, 16, 0, B, G0), true, false, n0));
    URC(layer_backward(u, 8, tv(u->dx0c, 16, 0, B, G0), tv(u->x0c, 16, 0, B, G0), tv(u->cat0, 48, 0, B, G0),
                       tv(u->dcat0, 48, 0, B, G0), true, false, n0));
    k_upsample_grad<<<blocks_for(n1 * 8, 256), 256, 0, s>>>(tv(u->dcat0, 48, 0, B, G0), tv(u->dx1d, 32, 0, B, G1), 32);
    ULAUNCH();
    URC(layer_backward(u, 7, tv(u->dx1d, 32, 0, B, G1), tv(u->x1d, 32, 0, B, G1), tv(u->x1c, 32, 0, B, G1),
                       tv(u->dx1c, 32, 0, B, G1), true, false, n1));
    URC(layer_backward(u, 6, tv(u->dx1c, 32, 0, B, G1), tv(u->x1c, 32, 0, B, G1), tv(u->cat1, 96, 0, B, G1),
                       tv(u->dcat1, 96, 0, B, G1), true, false, n1));
    k_upsample_grad<<<blocks_for(n2 * 16, 256), 256, 0, s>>>(tv(u->dcat1, 96, 0, B, G1), tv(u->dx2b, 64, 0, B, G2), 64);
    ULAUNCH();
    URC(layer_backward(u, 5, tv(u->dx2b, 64, 0, B, G2), tv(u->x2b, 64, 0, B, G2), tv(u->x2a, 64, 0, B, G2),
                       tv(u->dx2a, 64, 0, B, G2), true, false, n2));
    URC(layer_backward(u, 4, tv(u->dx2a, 64, 0, B, G2), tv(u->x2a, 64, 0, B, G2), tv(u->p2, 32, 0, B, G2),
                       tv(u->dp2, 32, 0, B, G2), true, false, n2));
    k_pool_grad<<<blocks_for(n2 * 8, 256), 256, 0, s>>>(tv(u->dp2, 32, 0, B, G2), tv(u->dcat1, 96, 64, B, G1), 32);
    ULAUNCH();
    URC(layer_backward(u, 3, tv(u->dcat1, 96, 64, B, G1), tv(u->cat1, 96, 64, B, G1), tv(u->x1a, 32, 0, B, G1),
                       tv(u->dx1a, 32, 0, B, G1), true, false, n1));
    URC(layer_backward(u, 2, tv(u->dx1a, 32, 0, B, G1), tv(u->x1a, 32, 0, B, G1), tv(u->p1, 16, 0, B, G1),
                       tv(u->dp1, 16, 0, B, G1), true, false, n1));
    k_pool_grad<<<blocks_for(n1 * 4, 256), 256, 0, s>>>(tv(u->dp1, 16, 0, B, G1), tv(u->dcat0, 48, 32, B, G0), 16);
    ULAUNCH();
    URC(layer_backward(u, 1, tv(u->dcat0, 48, 32, B, G0), tv(u->cat0, 48, 32, B, G0), tv(u->x0a, 16, 0, B, G0),
                       tv(u->dx0a, 16, 0, B, G0), true, false, n0));
    URC(layer_backward(u, 0, tv(u->dx0a, 16, 0, B, G0), tv(u->x0a, 16, 0, B, G0), tv(u->in, 16, 0, B, G0), none,
                       false, false, n0));
    return PLATO_OK;
}

}  // namespace

extern "C" {

const char* plato_unet_last_error(void) { return g_unet_error.c_str(); }

int plato_unet_create(const int32_t nodes[3], int32_t max_batch, plato_unet** out) {
    if (!out) return fail(PLATO_BAD_INPUT, "null output pointer");
    *out = nullptr;
    if (!nodes || max_batch < 1) return fail(PLATO_BAD_INPUT, "node grid and max_batch >= 1 required");
    for (int d = 0; d < 3; ++d)
        if (nodes[d] < 2 || nodes[d] > 4096) return fail(PLATO_BAD_INPUT, "node grid extents must be in [2, 4096]");
    plato_unet* u = new plato_unet();
    u->max_batch = max_batch;
    for (int d = 0; d < 3; ++d) {
        u->n[d] = nodes[d];
        u->g0[d] = (nodes[d] + 3) / 4 * 4;
    }
    if (halo_elems(u->g0, max_batch, 1) >= (int64_t(1) << 31)) {
        delete u;
        return fail(PLATO_BAD_INPUT, "node grid x max_batch too large (2^31 haloed positions at most)");
    }
    // layers: {cin, cout, taps, relu}
    const int spec[11][4] = {{16, 16, 27, 1}, {16, 16, 27, 1}, {16, 32, 27, 1}, {32, 32, 27, 1}, {32, 64, 27, 1},
                             {64, 64, 27, 1}, {96, 32, 27, 1}, {32, 32, 27, 1}, {48, 16, 27, 1}, {16, 16, 27, 1},
                             {16, 9, 1, 0}};
    int64_t off = 0;
    for (auto& sp : spec) {
        Layer L;
        L.cin = sp[0];
        L.cout = sp[1];
        L.taps = sp[2];
        L.relu = sp[3];
        L.w_off = off;
        off += int64_t(L.taps) * L.cout * L.cin;
        L.b_off = off;
        off += L.cout;
        u->layers.push_back(L);
    }
    u->nparams = off;
    auto cleanup = [&](int rc) {
        std::string msg = g_unet_error;
        plato_unet_destroy(u);
        g_unet_error = msg;
        return rc;
    };
#define CA(p, n)                               \
    do {                                       \
        int _rc = alloc(u, &(p), (n));         \
        if (_rc) return cleanup(_rc);          \
    } while (0)
    for (Layer& L : u->layers) {
        CA(L.wf, int64_t(L.taps) * L.coutp() * L.cin);
        CA(L.wb, int64_t(L.taps) * L.cin * (L.taps == 1 ? 16 : L.coutp()));
    }
    CA(u->params, u->nparams);
    CA(u->grads, u->nparams);
    CA(u->adam_m, u->nparams);
    CA(u->adam_v, u->nparams);
    const int B = max_batch;
    const int* G0 = u->g0;
    const int G1[3] = {G0[0] / 2, G0[1] / 2, G0[2] / 2};
    const int G2[3] = {G1[0] / 2, G1[1] / 2, G1[2] / 2};
    CA(u->in, halo_elems(G0, B, 16));
    CA(u->x0a, halo_elems(G0, B, 16));
    CA(u->cat0, halo_elems(G0, B, 48));
    CA(u->p1, halo_elems(G1, B, 16));
    CA(u->x1a, halo_elems(G1, B, 32));
    CA(u->cat1, halo_elems(G1, B, 96));
    CA(u->p2, halo_elems(G2, B, 32));
    CA(u->x2a, halo_elems(G2, B, 64));
    CA(u->x2b, halo_elems(G2, B, 64));
    CA(u->x1c, halo_elems(G1, B, 32));
    CA(u->x1d, halo_elems(G1, B, 32));
    CA(u->x0c, halo_elems(G0, B, 16));
    CA(u->x0d, halo_elems(G0, B, 16));
    CA(u->out, halo_elems(G0, B, 16));
    CA(u->dx0a, halo_elems(G0, B, 16));
    CA(u->dcat0, halo_elems(G0, B, 48));
    CA(u->dp1, halo_elems(G1, B, 16));
    CA(u->dx1a, halo_elems(G1, B, 32));
    CA(u->dcat1, halo_elems(G1, B, 96));
    CA(u->dp2, halo_elems(G2, B, 32));
    CA(u->dx2a, halo_elems(G2, B, 64));
    CA(u->dx2b, halo_elems(G2, B, 64));
    CA(u->dx1c, halo_elems(G1, B, 32));
    CA(u->dx1d, halo_elems(G1, B, 32));
    CA(u->dx0c, halo_elems(G0, B, 16));
    CA(u->dx0d, halo_elems(G0, B, 16));
    CA(u->mbuf, halo_elems(G0, B, 64) > halo_elems(G1, B, 64) ? halo_elems(G0, B, 64) : halo_elems(G1, B, 64));
    CA(u->loss_d, 1);
    CA(u->conv_err, 1);
#undef CA
    *out = u;
    return PLATO_OK;
}

int plato_unet_destroy(plato_unet* u) {
    if (!u) return PLATO_OK;
    if (u->stream) cudaStreamSynchronize(u->stream);
    for (void* p : u->allocs) cudaFree(p);
    delete u;
    return PLATO_OK;
}

int plato_unet_set_conv_kernel(plato_unet* u, int32_t kind) {
    if (!u) return fail(PLATO_BAD_INPUT, "null network");
    if (kind != PLATO_UNET_CONV_TCGEN05 && kind != PLATO_UNET_CONV_MMA_SYNC)
        return fail(PLATO_BAD_INPUT, "unknown convolution kernel kind");
    u->conv_kind = kind;
    return PLATO_OK;
}

int plato_unet_check(plato_unet* u) {
    if (!u) return fail(PLATO_BAD_INPUT, "null network");
    int err = 0;
    UCUDA(cudaMemcpyAsync(&err, u->conv_err, sizeof(int), cudaMemcpyDeviceToHost, u->stream));
    UCUDA(cudaStreamSynchronize(u->stream));
    if (err) {
        UCUDA(cudaMemsetAsync(u->conv_err, 0, sizeof(int), u->stream));
        return fail(PLATO_DEVICE_TIMEOUT, "a tensor-core convolution gave up waiting for its MMAs");
    }
    return PLATO_OK;
}

int plato_unet_set_stream(plato_unet* u, void* stream) {
    if (!u) return fail(PLATO_BAD_INPUT, "null network");
    u->stream = static_cast<cudaStream_t>(stream);
    return PLATO_OK;
}

int plato_unet_num_params(const plato_unet* u, int64_t* n) {
    if (!u || !n) return fail(PLATO_BAD_INPUT, "null argument");
    *n = u->nparams;
    return PLATO_OK;
}

int plato_unet_set_params(plato_unet* u, const float* params) {
    if (!u || !params) return fail(PLATO_BAD_INPUT, "null argument");
    UCUDA(cudaMemcpyAsync(u->params, params, sizeof(float) * size_t(u->nparams), cudaMemcpyDeviceToDevice, u->stream));
    UCUDA(cudaMemsetAsync(u->adam_m, 0, sizeof(float) * size_t(u->nparams), u->stream));
    UCUDA(cudaMemsetAsync(u->adam_v, 0, sizeof(float) * size_t(u->nparams), u->stream));
    return pack_all_weights(u);
}

int plato_unet_get_params(const plato_unet* u, float* params) {
    if (!u || !params) return fail(PLATO_BAD_INPUT, "null argument");
    UCUDA(cudaMemcpyAsync(params, u->params, sizeof(float) * size_t(u->nparams), cudaMemcpyDeviceToDevice, u->stream));
    return PLATO_OK;
}

int plato_unet_forward(plato_unet* u, int32_t batch, const float* input, float* output) {
    if (!u || !input || !output) return fail(PLATO_BAD_INPUT, "null argument");
    if (batch < 1 || batch > u->max_batch) return fail(PLATO_BAD_INPUT, "batch outside [1, max_batch]");
    URC(forward(u, batch, input));
    const int64_t nn = int64_t(batch) * u->n[0] * u->n[1] * u->n[2];
    k_unpack_output<<<blocks_for(nn * 9, 256), 256, 0, u->stream>>>(tv(u->out, 16, 0, batch, u->g0), u->n[0], u->n[1],
                                                                     u->n[2], output);
    ULAUNCH();
    return PLATO_OK;
}

int plato_unet_loss_and_gradients(plato_unet* u, int32_t batch, const float* input, const float* target,
                                  double* loss, float* grads) {
    if (!u || !input || !target) return fail(PLATO_BAD_INPUT, "null argument");
    if (batch < 1 || batch > u->max_batch) return fail(PLATO_BAD_INPUT, "batch outside [1, max_batch]");
    URC(forward(u, batch, input));
    cudaStream_t s = u->stream;
    UCUDA(cudaMemsetAsync(u->loss_d, 0, sizeof(double), s));
    UCUDA(cudaMemsetAsync(u->mbuf, 0, sizeof(bf16) * size_t(halo_elems(u->g0, batch, 16)), s));
    const int64_t n0 = int64_t(batch) * u->g0[0] * u->g0[1] * u->g0[2];
    k_loss<<<blocks_for(n0, 256), 256, 0, s>>>(tv(u->out, 16, 0, batch, u->g0), target, u->n[0], u->n[1], u->n[2],
                                                   tv(u->mbuf, 16, 0, batch, u->g0), u->loss_d);
    ULAUNCH();
    URC(backward(u, batch));
    if (grads)
        UCUDA(cudaMemcpyAsync(grads, u->grads, sizeof(float) * size_t(u->nparams), cudaMemcpyDeviceToDevice, s));
    if (loss) {
        UCUDA(cudaMemcpyAsync(loss, u->loss_d, sizeof(double), cudaMemcpyDeviceToHost, s));
        return plato_unet_check(u);  // synchronises the stream
    }
    return PLATO_OK;
}

int plato_unet_adam_step(plato_unet* u, float lr, int32_t step) {
    if (!u || step < 1 || !(lr > 0.f)) return fail(PLATO_BAD_INPUT, "adam needs a network, step >= 1 and lr > 0");
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.f - std::pow(b1, float(step)), c2 = 1.f - std::pow(b2, float(step));
    k_adam<<<blocks_for(u->nparams, 256), 256, 0, u->stream>>>(u->nparams, u->params, u->grads, u->adam_m, u->adam_v, lr,
                                                               b1, b2, 1e-8f, c1, c2);
    ULAUNCH();
    return pack_all_weights(u);
}

int plato_box_resample(const int32_t src_nodes[3], const int32_t dst_nodes[3], int32_t channels, const double* src,
                       double* dst, void* stream) {
    if (!src_nodes || !dst_nodes || !src || !dst || channels < 1) return fail(PLATO_BAD_INPUT, "bad resample arguments");
    for (int d = 0; d < 3; ++d)
        if (src_nodes[d] < 1 || dst_nodes[d] < 1) return fail(PLATO_BAD_INPUT, "node grid extents must be >= 1");
    const int64_t n = int64_t(dst_nodes[0]) * dst_nodes[1] * dst_nodes[2];
    k_box_resample<<<blocks_for(n, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        src_nodes[0], src_nodes[1], src_nodes[2], dst_nodes[0], dst_nodes[1], dst_nodes[2], channels, src, dst);
    ULAUNCH();
    return PLATO_OK;
}

int plato_unet_features(const int32_t src_nodes[3], const double* z, const int32_t net_nodes[3], float* features,
                        void* stream) {
    if (!src_nodes || !net_nodes || !z || !features) return fail(PLATO_BAD_INPUT, "bad feature arguments");
    const int64_t n = int64_t(net_nodes[0]) * net_nodes[1] * net_nodes[2];
    k_features<<<blocks_for(n, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        src_nodes[0], src_nodes[1], src_nodes[2], z, net_nodes[0], net_nodes[1], net_nodes[2], features);
    ULAUNCH();
    return PLATO_OK;
}

int plato_unet_subspace(const int32_t net_nodes[3], const float* output, const int32_t dst_nodes[3], double* W,
                        void* stream) {
    if (!net_nodes || !dst_nodes || !output || !W) return fail(PLATO_BAD_INPUT, "bad subspace arguments");
    const int64_t n = int64_t(dst_nodes[0]) * dst_nodes[1] * dst_nodes[2];
    k_subspace<<<blocks_for(n, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        net_nodes[0], net_nodes[1], net_nodes[2], output, dst_nodes[0], dst_nodes[1], dst_nodes[2], W);
    ULAUNCH();
    return PLATO_OK;
}

int plato_box_smooth(const int32_t nodes[3], int32_t channels, int32_t passes, float* data, float* scratch,
                     void* stream) {
    if (!nodes || !data || !scratch || channels < 1 || passes < 0) return fail(PLATO_BAD_INPUT, "bad smoothing arguments");
    const int64_t n = int64_t(nodes[0]) * nodes[1] * nodes[2] * channels;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    for (int p = 0; p < passes; ++p) {
        k_box_smooth<<<blocks_for(n, 256), 256, 0, s>>>(nodes[0], nodes[1], nodes[2], channels, data, scratch);
        ULAUNCH();
        UCUDA(cudaMemcpyAsync(data, scratch, sizeof(float) * size_t(n), cudaMemcpyDeviceToDevice, s));
    }
    return PLATO_OK;
}

}  // extern "C"
