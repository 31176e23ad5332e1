// pm_mlp.cu -- learned radiance cache kernels (see pm_mlp.cuh).
//
// Tensor-core path (sm_100a): tcgen05.mma.cta_group::1.kind::f16 with BF16
// operands read from shared memory through matrix descriptors and FP32
// accumulators in tensor memory (TMEM), issued by one thread, completion
// signalled through tcgen05.commit on an mbarrier, accumulators read back with
// tcgen05.ld (32 lanes x 32 bits per warp).
//
// Every operand lives in shared memory in the no-swizzle canonical layout of
// 8 x 8 core matrices (8 rows of 16 bytes), column blocks outermost:
//   (r, c) of an R-row matrix -> ((c / 8) * (R / 8) + r / 8) * 128 + (r % 8) * 16 + (c % 8) * 2.
// The same bytes serve as a K-major operand (rows = M or N, columns = K:
// leading byte offset 16 R between K blocks, stride byte offset 128 between
// row blocks) and as an MN-major operand (rows = K, columns = M or N: leading
// byte offset 128, stride byte offset 16 R).  So activations [sample][feature]
// feed the forward product (K-major A) and the weight gradient (MN-major A),
// output gradients [sample][out] feed the input gradient (K-major A) and the
// weight gradient (MN-major B), and weights [out][in] feed the forward product
// (K-major B) and the input gradient (MN-major B) without any copy.
//
// Per 128-sample tile (one thread per sample row, one warpgroup):
//   forward   D[128 x out] = X_l[128 x 64] W_l^T               M=128, 4 MMAs (K=16)
//   backward  dW_l += X_l^T[64 x 128] dY_l[128 x out]         M=64,  8 MMAs, accumulated in TMEM over tiles
//             dX   = dY_l[128 x out] W_l[out x 64]             M=128, out/16 MMAs
// Training runs TRAIN_GROUPS such tile pipelines per CTA (one warpgroup each,
// its own activation and gradient tiles, mbarrier and 64 TMEM columns), which
// all accumulate into the CTA's one set of weight-gradient columns: the chain
// of one tile is a series of small dependent products, so a second chain keeps
// the tensor pipe busy while the first one's epilogue runs.
// TMEM columns (training): [64 l, 64 l + out_l) the weight-gradient
// accumulator of layer l (M=64: rows 16 w + i in lanes 32 w + i), zeroed at
// the start; [TRAIN_FWD_COL + 64 g, +64) group g's forward / input-gradient tile.
#include <cmath>
#include <algorithm>
#include "pm_mlp.cuh"
#include "pm_device.cuh"

namespace pm {

namespace {

constexpr int TILE = 128;
constexpr int WAIT_LIMIT = 1 << 24;        // polls of an mbarrier before giving up
constexpr uint32_t TMEM_COLS_TRAIN = 512;
constexpr uint32_t TMEM_COLS_INFER = 256;   // 64 per warpgroup
constexpr uint32_t TRAIN_DW_COLS = 4 * 64 + MLP_OUT;   // weight-gradient accumulators of the five layers
constexpr uint32_t TRAIN_FWD_COL = 320;                // first per-group tile column

// shared-memory carve-up (bytes)
constexpr uint32_t W_BYTES = 4 * 8192 + 2048;       // layers 0-3: 64x64, layer 4: 16x64
constexpr uint32_t X_BYTES = TILE * MLP_DIM * 2;    // one [128][64] activation / gradient tile
// training: per group X_0 .. X_4 and one gradient tile (dY_l, replaced in
// place by dY_{l-1} once the products reading it have landed)
constexpr int TRAIN_GROUPS = 2;
constexpr int TRAIN_THREADS = 128 * TRAIN_GROUPS;
constexpr uint32_t TRAIN_GROUP_BYTES = 6 * X_BYTES;
constexpr uint32_t TRAIN_OFF_X = W_BYTES;
constexpr uint32_t TRAIN_OFF_BAR = TRAIN_OFF_X + TRAIN_GROUPS * TRAIN_GROUP_BYTES;
constexpr uint32_t TRAIN_SMEM = TRAIN_OFF_BAR + 64;
static_assert(TRAIN_SMEM <= 232448, "training tiles exceed the shared memory of a CTA");
static_assert(TRAIN_FWD_COL >= TRAIN_DW_COLS && TRAIN_FWD_COL + 64 * TRAIN_GROUPS <= TMEM_COLS_TRAIN, "TMEM layout");
// inference: INFER_GROUPS independent 128-row pipelines (one warpgroup each)
// share the weights; each owns one activation tile (the layers run in place),
// one mbarrier and 64 TMEM columns
constexpr int INFER_GROUPS = 4;
constexpr int INFER_THREADS = 128 * INFER_GROUPS;
constexpr uint32_t INFER_OFF_X = W_BYTES;
constexpr uint32_t INFER_OFF_BAR = INFER_OFF_X + INFER_GROUPS * X_BYTES;
constexpr uint32_t INFER_SMEM = INFER_OFF_BAR + 8 * INFER_GROUPS + 16;
static_assert(2 * (INFER_SMEM + 1024) <= 233472, "two inference CTAs per SM must fit in shared memory");

__host__ __device__ constexpr uint32_t w_off(int l) { return (uint32_t)l * 8192u; }

__device__ __forceinline__ uint32_t cm_off(int r, int c, int R) {
    return (uint32_t)(((c >> 3) * (R >> 3) + (r >> 3)) * 128 + (r & 7) * 16 + (c & 7) * 2);
}

// shared-memory matrix descriptor: start address, leading / stride byte
// offsets (16-byte units), descriptor version 1, no swizzle
__device__ __forceinline__ uint64_t sdesc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((saddr >> 4) & 0x3fffu) | ((uint64_t)((lbo >> 4) & 0x3fffu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3fffu) << 32) | ((uint64_t)1 << 46);
}

// instruction descriptor, kind::f16: FP32 accumulator, BF16 A and B
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N, int a_mn, int b_mn) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)a_mn << 15) | ((uint32_t)b_mn << 16) |
           ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void umma(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n"
        :: "r"(tmem_d), "l"(a), "l"(b), "r"(idesc), "r"(acc) : "memory");
}
__device__ __forceinline__ void umma_commit(uint64_t* bar) {
    const uint32_t a = (uint32_t)__cvta_generic_to_shared(bar);
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" :: "r"(a) : "memory");
}
__device__ __forceinline__ void mbar_init(uint64_t* bar) {
    const uint32_t a = (uint32_t)__cvta_generic_to_shared(bar);
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"(a) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
// bounded wait for the completion of phase `phase`; false on timeout
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t phase) {
    const uint32_t a = (uint32_t)__cvta_generic_to_shared(bar);
    for (int it = 0; it < WAIT_LIMIT; it++) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done) : "r"(a), "r"(phase) : "memory");
        if (done) return true;
    }
    return false;
}
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void tc_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// barrier `id` (1..4) over the 128 threads of one warpgroup; true iff v on all
// of them.  The id is an immediate in each branch, so the kernel reserves only
// the barriers it names (a register id reserves all 16 of the CTA).
template <int ID>
__device__ __forceinline__ uint32_t wg_red_and(uint32_t v) {
    uint32_t r;
    asm volatile(
        "{\n\t.reg .pred p, q;\n\tsetp.ne.u32 p, %1, 0;\n\t"
        "bar.red.and.pred q, %2, 128, p;\n\tselp.u32 %0, 1, 0, q;\n\t}\n"
        : "=r"(r) : "r"(v), "n"(ID) : "memory");
    return r;
}
__device__ __forceinline__ bool wg_sync_and(int id, bool v) {
    const uint32_t u = (uint32_t)v;
    uint32_t r;
    switch (id) {
        case 1: r = wg_red_and<1>(u); break;
        case 2: r = wg_red_and<2>(u); break;
        case 3: r = wg_red_and<3>(u); break;
        default: r = wg_red_and<4>(u); break;
    }
    return r != 0;
}

__device__ __forceinline__ void tmem_alloc(uint32_t* slot, uint32_t cols) {   // whole warp
    const uint32_t dst = (uint32_t)__cvta_generic_to_shared(slot);
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" :: "r"(dst), "r"(cols) : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t cols) {   // whole warp
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" :: "r"(taddr), "r"(cols) : "memory");
}
// 16 consecutive 32-bit columns of this thread's TMEM lane
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; i++) v[i] = __uint_as_float(r[i]);
}

// 64 consecutive 32-bit columns of this thread's TMEM lane, one wait
__device__ __forceinline__ void tmem_ld64(uint32_t taddr, float* v) {
    uint32_t r[64];
#define PM_R8(b) "=r"(r[b]), "=r"(r[b + 1]), "=r"(r[b + 2]), "=r"(r[b + 3]), "=r"(r[b + 4]), "=r"(r[b + 5]), \
                 "=r"(r[b + 6]), "=r"(r[b + 7])
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x64.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31,%32,%33,%34,%35,%36,%37,%38,%39,"
        "%40,%41,%42,%43,%44,%45,%46,%47,%48,%49,%50,%51,%52,%53,%54,%55,%56,%57,%58,%59,%60,%61,%62,%63}, [%64];"
        : PM_R8(0), PM_R8(8), PM_R8(16), PM_R8(24), PM_R8(32), PM_R8(40), PM_R8(48), PM_R8(56)
        : "r"(taddr));
#undef PM_R8
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 64; i++) v[i] = __uint_as_float(r[i]);
}
// zeros into 16 consecutive 32-bit columns of this thread's TMEM lane
__device__ __forceinline__ void tmem_zero16(uint32_t taddr) {
    const uint32_t z = 0u;
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1};"
        :: "r"(taddr), "r"(z) : "memory");
}

__device__ __forceinline__ uint32_t pack_bf16(float a, float b) {
    const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
    return *reinterpret_cast<const uint32_t*>(&h);
}
__device__ __forceinline__ void unpack_bf16(uint32_t u, float& a, float& b) {
    const __nv_bfloat162 h = *reinterpret_cast<const __nv_bfloat162*>(&u);
    a = __low2float(h);
    b = __high2float(h);
}

// weights (global [layer][out][in] bf16) -> core-matrix layout
__device__ void load_weights(const __nv_bfloat16* __restrict__ w, unsigned char* sW) {
    constexpr int CHUNKS = (4 * 64 + 16) * 8;   // 16-byte chunks
    for (int q = threadIdx.x; q < CHUNKS; q += blockDim.x) {
        const int row = q >> 3, j = q & 7;                  // global row over all layers, 8-column block
        const int l = row < 256 ? row >> 6 : 4;
        const int o = row < 256 ? row & 63 : row - 256;
        const uint4 v = *reinterpret_cast<const uint4*>(w + (size_t)l * MLP_LAYER_STRIDE + o * MLP_DIM + 8 * j);
        *reinterpret_cast<uint4*>(sW + w_off(l) + cm_off(o, 8 * j, mlp_out_dim(l))) = v;
    }
}

// one input sample: position, normal, whether it is used
// (sample i of cnt; base: array offset of sample 0 in pos3 / nrm3)
__device__ __forceinline__ bool load_sample(const MlpInputs& in, int64_t cnt, int64_t base, int64_t i, V3& p, V3& n) {
    p = v3(0.f, 0.f, 0.f);
    n = v3(0.f, 0.f, 1.f);
    if (i >= cnt) return false;
    if (in.pos3) {
        p = ld3(in.pos3 + 3 * (base + i));
        n = ld3(in.nrm3 + 3 * (base + i));
        return true;
    }
    const float4 a = in.rec_pos[i], b = in.rec_nrm[i];
    p = xyz(a);
    n = xyz(b);
    return (__float_as_uint(b.w) & in.flag_mask) != 0u;
}

// Encoding: u = (p - lo) * inv per axis, and the octahedral map of the normal
// to [0, 1]^2; each of the 5 values s gives sin(pi F 2^f s), cos(pi F 2^f s)
// for f = 0..5, F = freq0 (60 features, then 4 zeros).  Written as row `row` of an [128][64] tile.
// Octave 0 comes from sincospif, each further octave from the double-angle
// identities sin 2x = 2 sin x cos x, cos 2x = (cos x - sin x)(cos x + sin x):
// the angle error doubles per octave, 2^5 x a few 1e-8 after five, far below
// the BF16 rounding (2^-9 relative) the features then get.
__device__ __forceinline__ void write_features(unsigned char* sX, int row, const MlpNet& net, V3 p, V3 n) {
    float s[5];
    s[0] = (p.x - net.lo[0]) * net.inv[0];
    s[1] = (p.y - net.lo[1]) * net.inv[1];
    s[2] = (p.z - net.lo[2]) * net.inv[2];
    float a = fabsf(n.x) + fabsf(n.y) + fabsf(n.z);
    if (!(a > 0.f)) a = 1.f;
    float ox = n.x / a, oy = n.y / a;
    if (n.z < 0.f) {
        const float tx = (1.f - fabsf(oy)) * (ox >= 0.f ? 1.f : -1.f);
        const float ty = (1.f - fabsf(ox)) * (oy >= 0.f ? 1.f : -1.f);
        ox = tx;
        oy = ty;
    }
    s[3] = 0.5f * ox + 0.5f;
    s[4] = 0.5f * oy + 0.5f;
    // word w = 6 j + f holds features 2w, 2w + 1; each 8-feature block goes
    // to shared memory as soon as its four words exist
    uint32_t pk[4];
#pragma unroll
    for (int j = 0; j < 5; j++) {
        float sn, cs;
        sincospif(s[j] * net.freq0, &sn, &cs);
#pragma unroll
        for (int f = 0; f < 6; f++) {
            if (f > 0) {
                const float s2 = 2.f * sn * cs;
                const float c2 = (cs - sn) * (cs + sn);
                sn = s2;
                cs = c2;
            }
            const int w = 6 * j + f;
            pk[w & 3] = pack_bf16(sn, cs);
            if ((w & 3) == 3)
                *reinterpret_cast<uint4*>(sX + cm_off(row, 2 * (w - 3), TILE)) = make_uint4(pk[0], pk[1], pk[2], pk[3]);
        }
    }
    *reinterpret_cast<uint4*>(sX + cm_off(row, 56, TILE)) = make_uint4(pk[0], pk[1], 0u, 0u);
}

// forward product of layer l into TMEM columns [0, out)
__device__ __forceinline__ void issue_forward(int l, uint32_t tm, uint32_t xa, uint32_t wa) {
    const int out = mlp_out_dim(l);
    const uint32_t lbo_w = 16u * (uint32_t)out;
    const uint32_t id = idesc_bf16(TILE, out, 0, 0);
#pragma unroll
    for (int s = 0; s < 4; s++) umma(tm, sdesc(xa + 4096u * s, 2048u, 128u), sdesc(wa + 2u * lbo_w * s, lbo_w, 128u), id, s > 0);
}

// ReLU of a [128 x 64] TMEM tile row (this thread's) -> bf16 row of the next
// activation tile.  COLS columns per TMEM load (64: one wait per row, for
// kernels with the registers; 16: four loads, for the 64-register inference).
template <int COLS>
__device__ __forceinline__ void relu_row_to_smem(uint32_t taddr, unsigned char* dst, int row) {
#pragma unroll
    for (int c0 = 0; c0 < 64; c0 += COLS) {
        float v[COLS];
        if constexpr (COLS == 64) tmem_ld64(taddr + c0, v);
        else tmem_ld16(taddr + c0, v);
#pragma unroll
        for (int b = 0; b < COLS / 8; b++) {
            uint4 q;
            q.x = pack_bf16(fmaxf(v[8 * b + 0], 0.f), fmaxf(v[8 * b + 1], 0.f));
            q.y = pack_bf16(fmaxf(v[8 * b + 2], 0.f), fmaxf(v[8 * b + 3], 0.f));
            q.z = pack_bf16(fmaxf(v[8 * b + 4], 0.f), fmaxf(v[8 * b + 5], 0.f));
            q.w = pack_bf16(fmaxf(v[8 * b + 6], 0.f), fmaxf(v[8 * b + 7], 0.f));
            *reinterpret_cast<uint4*>(dst + cm_off(row, c0 + 8 * b, TILE)) = q;
        }
    }
}

// dY_{l-1} = dX * [X_l > 0] for this thread's row: dX from its TMEM lane, the
// mask from row `row` of X_l, the result (bf16) over the same row of g
__device__ __forceinline__ void masked_grad_row(uint32_t taddr, const unsigned char* xrow, unsigned char* g, int row) {
    float v[64];
    tmem_ld64(taddr, v);
#pragma unroll
    for (int b = 0; b < 8; b++) {
        const uint4 xq = *reinterpret_cast<const uint4*>(xrow + cm_off(row, 8 * b, TILE));
        const uint32_t xs[4] = {xq.x, xq.y, xq.z, xq.w};
        uint32_t o[4];
#pragma unroll
        for (int e = 0; e < 4; e++) {
            float x0, x1;
            unpack_bf16(xs[e], x0, x1);
            o[e] = pack_bf16(x0 > 0.f ? v[8 * b + 2 * e] : 0.f, x1 > 0.f ? v[8 * b + 2 * e + 1] : 0.f);
        }
        *reinterpret_cast<uint4*>(g + cm_off(row, 8 * b, TILE)) = make_uint4(o[0], o[1], o[2], o[3]);
    }
}

// Training: warpgroup g of the CTA runs its own tiles (g + G * CTA, then
// strided by G * grid): features, five forward products, the output gradient,
// then per layer (last first) the weight-gradient product into the CTA's
// shared accumulator and the input-gradient product, each waited on through
// the group's mbarrier.  Thread 0 of the group issues its products.  The
// accumulators are zeroed before any product; at the end the CTA adds them to
// the global gradient once.
__global__ void __launch_bounds__(TRAIN_THREADS, 1)
k_mlp_train(MlpNet net, MlpInputs in, const float* __restrict__ target, const float* __restrict__ weight,
            float grad_scale, float* __restrict__ grad, float* __restrict__ loss_sum, unsigned* status) {
    extern __shared__ __align__(1024) unsigned char smem[];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int g = tid >> 7, row = tid & 127;
    unsigned char* sW = smem;
    unsigned char* sX = smem + TRAIN_OFF_X + g * TRAIN_GROUP_BYTES;   // X_0 .. X_4
    unsigned char* sG = sX + 5 * X_BYTES;                             // the gradient tile
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem + TRAIN_OFF_BAR);
    uint64_t* bar = bars + g;
    uint32_t* tslot = reinterpret_cast<uint32_t*>(smem + TRAIN_OFF_BAR + 8 * TRAIN_GROUPS);
    load_weights(net.w, sW);
    if (tid < TRAIN_GROUPS) mbar_init(bars + tid);
    if (warp == 0) tmem_alloc(tslot, TMEM_COLS_TRAIN);
    fence_async_smem();
    tc_before();
    __syncthreads();
    tc_after();
    const uint32_t tbase = *tslot;
    const uint32_t my_lanes = (uint32_t)(32 * (warp & 3)) << 16;
    // zero the weight-gradient accumulators (group 0's four warps cover the 128 lanes)
    if (g == 0) {
#pragma unroll 1
        for (uint32_t c = 0; c < TRAIN_DW_COLS; c += 16) tmem_zero16(tbase + my_lanes + c);
        asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
    }
    tc_before();
    __syncthreads();
    tc_after();
    const uint32_t tm = tbase + TRAIN_FWD_COL + 64u * (uint32_t)g;   // this group's tile columns
    const uint32_t sW_a = (uint32_t)__cvta_generic_to_shared(sW);
    const uint32_t sX_a = (uint32_t)__cvta_generic_to_shared(sX);
    const uint32_t sG_a = (uint32_t)__cvta_generic_to_shared(sG);
    const bool leader = row == 0;
    const int bar_id = 1 + g;
    const float inv_scale = 1.f / net.out_scale;
    uint32_t phase = 0;
    bool ok = true;
    float loss = 0.f;
    const int64_t tiles = (in.n + TILE - 1) / TILE;
    int64_t base = in.base_dev ? *in.base_dev : 0;
    if (in.base_wrap > 0 && base + in.n > in.base_wrap) base = 0;
    const int64_t stride = (int64_t)gridDim.x * TRAIN_GROUPS;
    for (int64_t tile = (int64_t)blockIdx.x * TRAIN_GROUPS + g; tile < tiles && ok; tile += stride) {
        const int64_t i = tile * TILE + row;
        V3 p, n;
        const bool use = load_sample(in, in.n, base, i, p, n);
        const float wgt = use ? (weight ? weight[base + i] : 1.f) : 0.f;
        const V3 t = use ? ld3(target + 3 * (base + i)) : v3(0.f, 0.f, 0.f);
        write_features(sX, row, net, p, n);
        fence_async_smem();
        tc_before();
        wg_sync_and(bar_id, true);
        tc_after();
        float y[3] = {0.f, 0.f, 0.f};
        for (int l = 0; l < MLP_LAYERS && ok; l++) {
            if (leader) {
                issue_forward(l, tm, sX_a + l * X_BYTES, sW_a + w_off(l));
                umma_commit(bar);
            }
            const bool done = mbar_wait(bar, phase);
            phase ^= 1u;
            tc_after();
            if (done) {
                if (l < MLP_LAYERS - 1) {
                    relu_row_to_smem<64>(tm + my_lanes, sX + (l + 1) * X_BYTES, row);
                } else {
                    float v[16];
                    tmem_ld16(tm + my_lanes, v);
                    y[0] = v[0]; y[1] = v[1]; y[2] = v[2];
                }
            }
            tc_before();
            fence_async_smem();
            ok = wg_sync_and(bar_id, done);
            tc_after();
        }
        if (!ok) break;
        // d(loss)/dy for the MSE against target / out_scale
        const float d0 = y[0] - t.x * inv_scale, d1 = y[1] - t.y * inv_scale, d2 = y[2] - t.z * inv_scale;
        loss += wgt * (d0 * d0 + d1 * d1 + d2 * d2);
        const float gs = grad_scale * wgt;
        *reinterpret_cast<uint4*>(sG + cm_off(row, 0, TILE)) =
            make_uint4(pack_bf16(gs * d0, gs * d1), pack_bf16(gs * d2, 0.f), 0u, 0u);
        *reinterpret_cast<uint4*>(sG + cm_off(row, 8, TILE)) = make_uint4(0u, 0u, 0u, 0u);
        fence_async_smem();
        tc_before();
        wg_sync_and(bar_id, true);
        tc_after();
        for (int l = MLP_LAYERS - 1; l >= 0; l--) {
            const int out = mlp_out_dim(l);
            const uint32_t xa = sX_a + l * X_BYTES, wa = sW_a + w_off(l);
            if (leader) {
                const uint32_t idw = idesc_bf16(64, out, 1, 1);
#pragma unroll
                for (int s = 0; s < TILE / 16; s++)
                    umma(tbase + 64u * l, sdesc(xa + 256u * s, 128u, 2048u), sdesc(sG_a + 256u * s, 128u, 2048u), idw, 1u);
                if (l > 0) {
                    const uint32_t idx = idesc_bf16(TILE, 64, 0, 1);
                    for (int s = 0; s < out / 16; s++)
                        umma(tm, sdesc(sG_a + 4096u * s, 2048u, 128u), sdesc(wa + 256u * s, 128u, 16u * (uint32_t)out),
                             idx, s > 0);
                }
                umma_commit(bar);
            }
            const bool done = mbar_wait(bar, phase);
            phase ^= 1u;
            tc_after();
            // both products have read dY_l: dY_{l-1} replaces it
            if (done && l > 0) masked_grad_row(tm + my_lanes, sX + l * X_BYTES, sG, row);
            tc_before();
            fence_async_smem();
            ok = wg_sync_and(bar_id, done);
            tc_after();
            if (!ok) break;
        }
    }
    if (!ok) {
        if (leader) raise_status(status, ST_TIMEOUT);
        (void)mbar_wait(bar, phase ^ 1u);   // let the late product land before the columns are freed
    }
    tc_before();
    const bool all_ok = __syncthreads_and(ok) != 0;
    tc_after();
    if (all_ok && (int64_t)blockIdx.x * TRAIN_GROUPS < tiles) {
        // weight gradients: lanes 0-15 of each warp hold rows 16 (warp % 4) + lane
        // (input index); group g drains the layers l with l % TRAIN_GROUPS == g
        for (int l = g; l < MLP_LAYERS; l += TRAIN_GROUPS) {
            const int out = mlp_out_dim(l);
            for (int c0 = 0; c0 < out; c0 += 16) {
                float v[16];
                tmem_ld16(tbase + my_lanes + 64u * l + c0, v);
                if (lane < 16) {
                    const int m = 16 * (warp & 3) + lane;
#pragma unroll
                    for (int e = 0; e < 16; e++) atomicAdd(grad + (size_t)l * MLP_LAYER_STRIDE + (c0 + e) * MLP_DIM + m, v[e]);
                }
            }
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) loss += __shfl_xor_sync(0xffffffffu, loss, o);
    if (lane == 0 && loss != 0.f) atomicAdd(loss_sum, loss);
    tc_before();
    __syncthreads();
    tc_after();
    if (warp == 0) tmem_dealloc(tbase, TMEM_COLS_TRAIN);
}

// Inference: warpgroup g of the CTA runs its own tiles (g + G * CTA, then
// strided by G * grid) through the five layers; its 128 threads each own one
// sample row (row = TMEM lane), thread 0 of the group issues the products.
// Layer l's product reads the group's activation tile, and once its commit
// has landed that tile is free, so the ReLU output of layer l overwrites it in
// place.  The next tile's samples are loaded while the current one runs.
__global__ void __launch_bounds__(INFER_THREADS, 2)
k_mlp_infer(MlpNet net, MlpInputs in, float* __restrict__ out, unsigned* status) {
    extern __shared__ __align__(1024) unsigned char smem[];
    const int tid = threadIdx.x, warp = tid >> 5;
    const int g = tid >> 7, row = tid & 127;
    unsigned char* sW = smem;
    unsigned char* sX = smem + INFER_OFF_X + g * X_BYTES;
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem + INFER_OFF_BAR);
    uint64_t* bar = bars + g;
    uint32_t* tslot = reinterpret_cast<uint32_t*>(smem + INFER_OFF_BAR + 8 * INFER_GROUPS);
    load_weights(net.w, sW);
    if (tid < INFER_GROUPS) mbar_init(bars + tid);
    if (warp == 0) tmem_alloc(tslot, TMEM_COLS_INFER);
    fence_async_smem();
    tc_before();
    __syncthreads();
    tc_after();
    const uint32_t tm = *tslot + 64u * (uint32_t)g;
    const uint32_t my_lanes = (uint32_t)(32 * (warp & 3)) << 16;
    const uint32_t sW_a = (uint32_t)__cvta_generic_to_shared(sW);
    const uint32_t sX_a = (uint32_t)__cvta_generic_to_shared(sX);
    const bool leader = row == 0;
    const int bar_id = 1 + g;
    uint32_t phase = 0;
    bool ok = true;
    const int64_t cnt = in.n_dev ? (int64_t)min(*in.n_dev, (unsigned long long)in.n) : in.n;
    const int64_t tiles = (cnt + TILE - 1) / TILE;
    const int64_t stride = (int64_t)gridDim.x * INFER_GROUPS;
    int64_t tile = (int64_t)blockIdx.x * INFER_GROUPS + g;
    V3 p, n;
    bool use = load_sample(in, cnt, 0, tile * TILE + row, p, n);
    for (; tile < tiles && ok; tile += stride) {
        const int64_t i = tile * TILE + row;
        write_features(sX, row, net, p, n);
        const bool use_cur = use;
        use = load_sample(in, cnt, 0, (tile + stride) * TILE + row, p, n);   // next tile's sample, in flight
        fence_async_smem();
        tc_before();
        wg_sync_and(bar_id, true);
        tc_after();
        float y[3] = {0.f, 0.f, 0.f};
        for (int l = 0; l < MLP_LAYERS && ok; l++) {
            if (leader) {
                issue_forward(l, tm, sX_a, sW_a + w_off(l));
                umma_commit(bar);
            }
            const bool done = mbar_wait(bar, phase);
            phase ^= 1u;
            tc_after();
            if (done) {
                if (l < MLP_LAYERS - 1) {
                    relu_row_to_smem<16>(tm + my_lanes, sX, row);
                } else {
                    float v[16];
                    tmem_ld16(tm + my_lanes, v);
                    y[0] = v[0]; y[1] = v[1]; y[2] = v[2];
                }
            }
            tc_before();
            fence_async_smem();
            ok = wg_sync_and(bar_id, done);
            tc_after();
        }
        if (!ok) break;
        if (i < cnt) {
            const float sc = use_cur ? net.out_scale : 0.f;
            out[3 * i] = y[0] * sc;
            out[3 * i + 1] = y[1] * sc;
            out[3 * i + 2] = y[2] * sc;
        }
    }
    if (!ok) {
        if (leader) raise_status(status, ST_TIMEOUT);
        (void)mbar_wait(bar, phase ^ 1u);   // let the late product land before the columns are freed
    }
    tc_before();
    __syncthreads();
    tc_after();
    if (warp == 0) tmem_dealloc(*tslot, TMEM_COLS_INFER);
}

__device__ __forceinline__ void adam_update(int i, float* __restrict__ w32, __nv_bfloat16* __restrict__ w16,
                                            float* __restrict__ grad, float* __restrict__ m, float* __restrict__ v,
                                            float lr, float b1, float b2, float eps, float c1, float c2) {
    const float g = grad[i];
    const float mi = b1 * m[i] + (1.f - b1) * g;
    const float vi = b2 * v[i] + (1.f - b2) * g * g;
    m[i] = mi;
    v[i] = vi;
    const float w = w32[i] - lr * (mi * c1) / (sqrtf(vi * c2) + eps);
    w32[i] = w;
    w16[i] = __float2bfloat16_rn(w);
    grad[i] = 0.f;
}

__global__ void k_adam(float* __restrict__ w32, __nv_bfloat16* __restrict__ w16, float* __restrict__ grad,
                       float* __restrict__ m, float* __restrict__ v, float lr, float b1, float b2, float eps,
                       float c1, float c2) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < MLP_PARAMS) adam_update(i, w32, w16, grad, m, v, lr, b1, b2, eps, c1, c2);
}

__global__ void k_step_inc(int* step) { *step += 1; }

// k_adam with the bias corrections 1 / (1 - beta^step) formed on the device
__global__ void k_adam_dev(float* __restrict__ w32, __nv_bfloat16* __restrict__ w16, float* __restrict__ grad,
                           float* __restrict__ m, float* __restrict__ v, float lr, float b1, float b2, float eps,
                           const int* __restrict__ step) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= MLP_PARAMS) return;
    const int s = *step;
    const float c1 = (float)(1.0 / (1.0 - pow((double)b1, (double)s)));
    const float c2 = (float)(1.0 / (1.0 - pow((double)b2, (double)s)));
    adam_update(i, w32, w16, grad, m, v, lr, b1, b2, eps, c1, c2);
}

__global__ void k_to_bf16(const float* __restrict__ w32, __nv_bfloat16* __restrict__ w16) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < MLP_PARAMS) w16[i] = __float2bfloat16_rn(w32[i]);
}

}  // namespace

cudaError_t mlp_train(const MlpNet& net, const MlpInputs& in, const float* target, const float* weight,
                      float grad_scale, float* grad, float* loss_sum, unsigned* status, int sm_count,
                      cudaStream_t st) {
    if (in.n <= 0) return cudaSuccess;
    cudaError_t e = cudaFuncSetAttribute(k_mlp_train, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TRAIN_SMEM);
    if (e != cudaSuccess) return e;
    const int64_t tiles = (in.n + TILE - 1) / TILE;
    const int64_t ctas = (tiles + TRAIN_GROUPS - 1) / TRAIN_GROUPS;
    const int grid = (int)std::min<int64_t>(ctas, std::max(sm_count, 1));   // one CTA per SM: 512 TMEM columns each
    k_mlp_train<<<grid, TRAIN_THREADS, TRAIN_SMEM, st>>>(net, in, target, weight, grad_scale, grad, loss_sum, status);
    return cudaGetLastError();
}

cudaError_t mlp_infer(const MlpNet& net, const MlpInputs& in, float* out, unsigned* status, int sm_count,
                      cudaStream_t st) {
    if (in.n <= 0) return cudaSuccess;
    cudaError_t e = cudaFuncSetAttribute(k_mlp_infer, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)INFER_SMEM);
    if (e != cudaSuccess) return e;
    // Two CTAs per SM (8 tile pipelines): each holds 256 of the SM's 512 TMEM
    // columns, 64 registers x 512 threads (half the register file, the launch
    // bounds) and under half the shared memory, with the largest carve-out.
    // The occupancy calculator reports one CTA per SM for any kernel that
    // allocates TMEM, so the grid is sized from these limits instead; the
    // tile loop is strided over the whole grid either way.
    e = cudaFuncSetAttribute(k_mlp_infer, cudaFuncAttributePreferredSharedMemoryCarveout,
                             (int)cudaSharedmemCarveoutMaxShared);
    if (e != cudaSuccess) return e;
    const int per_sm = 512 / (int)TMEM_COLS_INFER;
    const int64_t tiles = (in.n + TILE - 1) / TILE;
    const int64_t ctas = (tiles + INFER_GROUPS - 1) / INFER_GROUPS;
    const int grid = (int)std::min<int64_t>(ctas, (int64_t)per_sm * std::max(sm_count, 1));
    k_mlp_infer<<<grid, INFER_THREADS, INFER_SMEM, st>>>(net, in, out, status);
    return cudaGetLastError();
}

cudaError_t mlp_adam(float* w32, __nv_bfloat16* w16, float* grad, float* m, float* v, int step, float lr,
                     float beta1, float beta2, float eps, cudaStream_t st) {
    const float c1 = (float)(1.0 / (1.0 - std::pow((double)beta1, step)));
    const float c2 = (float)(1.0 / (1.0 - std::pow((double)beta2, step)));
    k_adam<<<(MLP_PARAMS + 255) / 256, 256, 0, st>>>(w32, w16, grad, m, v, lr, beta1, beta2, eps, c1, c2);
    return cudaGetLastError();
}

cudaError_t mlp_adam_dev(float* w32, __nv_bfloat16* w16, float* grad, float* m, float* v, int* step_dev, float lr,
                         float beta1, float beta2, float eps, cudaStream_t st, bool increment) {
    if (increment) k_step_inc<<<1, 1, 0, st>>>(step_dev);
    k_adam_dev<<<(MLP_PARAMS + 255) / 256, 256, 0, st>>>(w32, w16, grad, m, v, lr, beta1, beta2, eps, step_dev);
    return cudaGetLastError();
}

cudaError_t mlp_to_bf16(const float* w32, __nv_bfloat16* w16, cudaStream_t st) {
    k_to_bf16<<<(MLP_PARAMS + 255) / 256, 256, 0, st>>>(w32, w16);
    return cudaGetLastError();
}

}  // namespace pm
