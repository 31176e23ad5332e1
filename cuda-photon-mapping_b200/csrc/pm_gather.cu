// pm_gather.cu -- kNN photon gather + radiance estimate.
//
// Reference: CudaPhotonMapping/PhotonGrid.cu:222-284 (cube of cells of half
// width ceil(r / cell) around the query's cell, distance test <= r),
// PhotonMaxHeap.cuh:43-127 (bounded max-heap of k), Raytracer.cuh:110-138
// (Gaussian-filtered density estimate over the selected photons).
//
// Selection rule: the k photons with the smallest (distance, source id) pairs
// among those with distance <= r.  This is the reference heap's set whenever no
// two candidates tie at the k-th distance; on ties it is deterministic (the
// reference's heap keeps whichever the sift order leaves).  Distances are the
// reference's length(p - q) in IEEE float, so the sets are bit-exact.
//
// One warp per query.  Photons are stored by (cell, sub-cell); the warp walks
// the query's sub-cell and the shell of sub-cells around it, then shells
// further out (nearest first), within the reference's cube of cells, skipping
// every sub-cell whose box lies farther than the current bound on the k-th
// distance (with a margin far above float rounding) and stopping at the first
// shell that lies entirely farther.  Non-empty sub-cells are queued and their
// photons scanned as one list, one photon per lane (one 16-byte load each):
// lanes test the squared distance against a bound slightly above the
// threshold's square, take the correctly rounded sqrt only for survivors, and
// append the survivors' 64-bit keys (distance bits << 32 | source id;
// non-negative float bits order like the floats, so integer order is the
// lexicographic order) to a per-warp shared-memory store by ballot, counting
// each in a 64-bin histogram of distance over [0, r] (over [0, g] once the
// first ring's density guess g bounds the stored distances).  After each shell the
// histogram bounds the k-th distance (the upper edge of the bin where the
// running count reaches k).  When the store fills, and at the end, the exact
// k-th key is found from the histogram: the keys of its bin (a handful) are
// sorted by the warp (an MSB-first radix select over the store when the bin
// holds more than 32), and the store is cut to the k best.  The answer is the
// exhaustive walk's.
#include <algorithm>
#include "pm_gather.cuh"
#include "pm_device.cuh"

namespace pm {

namespace {

constexpr int WARPS = 8;   // queries per block

constexpr int QCAP = 64;   // queued sub-cells per warp

// distance histogram bins over [0, r], or over [0, g] once the first ring's
// guess g is set: 64 for the frame's gather (its queries nearly all take the
// guess), 256 for the batch's (many of its queries take none, and 64 bins
// over [0, r] leave too many keys in the k-th bin)
constexpr int GATHER_BINS = 64;
constexpr int MULTI_BINS = 256;

template <int UCAP, int NB>
struct WarpStore {
    unsigned long long key[UCAP];
    uint32_t slot[UCAP];
    uint32_t hist[256];   // radix-select histogram; doubles as 32 x u64 scratch
    uint32_t dh[NB];      // distance histogram of the keys in the store
    unsigned long long sel[32];
    uint32_t qa[QCAP];    // queued sub-cells: first photon, photon count
    uint32_t qc[QCAP];
};

__device__ __forceinline__ unsigned long long shfl_u64(unsigned long long v, int src) {
    return __shfl_sync(0xffffffffu, v, src);
}
__device__ __forceinline__ unsigned long long shfl_xor_u64(unsigned long long v, int m) {
    return __shfl_xor_sync(0xffffffffu, v, m);
}

// ascending bitonic sort of one value per lane
__device__ __forceinline__ unsigned long long warp_sort32(unsigned long long v, int lane) {
#pragma unroll
    for (int size = 2; size <= 32; size <<= 1) {
#pragma unroll
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
            unsigned long long o = shfl_xor_u64(v, stride);
            bool ascending = (lane & size) == 0;
            bool lower = (lane & stride) == 0;
            unsigned long long lo = v < o ? v : o, hi = v < o ? o : v;
            v = (lower == ascending) ? lo : hi;
        }
    }
    return v;
}

// the need-th smallest (1-based) of U.key[0, n); need <= n; keys are unique.
// MSB-first radix select: the bits above the highest bit in which two keys
// differ are skipped, each round histograms the next (up to) 8 bits of the keys
// still in play (lanes with equal digits add once, __match_any_sync), and the
// round that leaves <= 32 keys finishes with a 32-lane bitonic sort.
template <int UCAP, int NB>
__device__ unsigned long long select_kth(WarpStore<UCAP, NB>& U, int n, int need, int lane) {
    unsigned long long* scratch = reinterpret_cast<unsigned long long*>(U.hist);
    const unsigned long long k0 = U.key[0];
    unsigned long long diff = 0ull;
    for (int i = lane; i < n; i += 32) diff |= U.key[i] ^ k0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) diff |= shfl_xor_u64(diff, o);
    if (diff == 0ull) return k0;
    int hi = 64 - __clzll((long long)diff);          // bits [hi, 64) are common to all keys
    unsigned long long mask = hi == 64 ? 0ull : ~0ull << hi;
    unsigned long long prefix = k0 & mask;
    while (true) {
        const int shift = hi > 8 ? hi - 8 : 0;
        const unsigned dmask = (1u << (hi - shift)) - 1u;
#pragma unroll
        for (int b = 0; b < 8; b++) U.hist[8 * lane + b] = 0u;
        __syncwarp();
        for (int base = 0; base < n; base += 32) {
            const int i = base + lane;
            const unsigned long long kk = i < n ? U.key[i] : 0ull;
            const bool m = i < n && (kk & mask) == prefix;
            const unsigned d = (unsigned)(kk >> shift) & dmask;
            const unsigned act = __ballot_sync(0xffffffffu, m);
            if (m) {
                const unsigned peers = __match_any_sync(act, d);
                if ((peers & lanemask_lt()) == 0u) atomicAdd(&U.hist[d], (uint32_t)__popc(peers));
            }
        }
        __syncwarp();
        uint32_t c[8], sum = 0;
#pragma unroll
        for (int b = 0; b < 8; b++) { c[b] = U.hist[8 * lane + b]; sum += c[b]; }
        uint32_t incl = sum;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += y;
        }
        const uint32_t excl = incl - sum;
        const unsigned own = __ballot_sync(0xffffffffu, excl < (uint32_t)need && (uint32_t)need <= incl);
        const int owner = own ? __ffs(own) - 1 : 0;
        int bin = 0;
        uint32_t before = 0, cnt = 0;
        if (lane == owner) {
            uint32_t run = excl;
#pragma unroll
            for (int b = 0; b < 8; b++) {
                if (cnt == 0 && (uint32_t)need <= run + c[b]) { bin = 8 * lane + b; before = run; cnt = c[b]; }
                run += c[b];
            }
        }
        bin = __shfl_sync(0xffffffffu, bin, owner);
        before = __shfl_sync(0xffffffffu, before, owner);
        cnt = __shfl_sync(0xffffffffu, cnt, owner);
        need -= (int)before;
        prefix |= (unsigned long long)bin << shift;
        mask |= (unsigned long long)dmask << shift;
        hi = shift;
        __syncwarp();
        if (cnt <= 32u || hi == 0) {
            // the few keys under this prefix: gather one per lane, sort, pick
            int got = 0;
            for (int base = 0; base < n; base += 32) {
                int i = base + lane;
                unsigned long long kk = i < n ? U.key[i] : ~0ull;
                bool m = i < n && (kk & mask) == prefix;
                unsigned bm = __ballot_sync(0xffffffffu, m);
                if (m) scratch[got + __popc(bm & lanemask_lt())] = kk;
                got += __popc(bm);
            }
            __syncwarp();
            unsigned long long v = lane < got ? scratch[lane] : ~0ull;
            __syncwarp();
            v = warp_sort32(v, lane);
            return shfl_u64(v, need - 1);
        }
    }
}

template <int UCAP, int NB>
__device__ __forceinline__ unsigned long long warp_max_key(const WarpStore<UCAP, NB>& U, int n, int lane) {
    unsigned long long m = 0ull;
    for (int i = lane; i < n; i += 32) m = U.key[i] > m ? U.key[i] : m;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        unsigned long long y = shfl_xor_u64(m, o);
        m = y > m ? y : m;
    }
    return m;
}

// Cell / sub-cell of a point: the quotient (p - min) / cell selects the cell
// (clamped, CudaPhotonMapping/PhotonGrid.cu:10-23); its fractional part the sub-cell.
__device__ __forceinline__ void locate(float p, float mn, float cell, int g, int S, int& c, int& s) {
    float u = (p - mn) / cell;
    c = min(max((int)u, 0), g - 1);
    float f = u - (float)c;
    s = min(max((int)(f * (float)S), 0), S - 1);
}

// distance from q to the slab [lo, hi] along one axis; an open side (photons
// clamped into a boundary cell from outside the grid) is at infinity
__device__ __forceinline__ float axis_gap(float q, float lo, float hi, bool open_lo, bool open_hi) {
    float a = open_lo ? 0.f : lo - q;
    float b = open_hi ? 0.f : q - hi;
    return fmax3(a, b, 0.f);
}

// u / d for 0 <= u < 2^22, d > 0: float estimate, one correction step
__device__ __forceinline__ int small_div(int u, int d, float inv) {
    int q = (int)(((float)u + 0.5f) * inv);
    const int r = u - q * d;
    if (r < 0) q--;
    else if (r >= d) q++;
    return q;
}

// Offsets of the t-th sub-cell of the shell at Chebyshev distance R around a
// sub-cell (side = 2R + 1; 2 side^2 + 4 (side - 1)(side - 2) members): the two
// full z faces, then the perimeter of each inner z layer.
__device__ __forceinline__ void shell_member(int t, int R, int side, float inv_side, float inv_per, int& dx,
                                             int& dy, int& dz) {
    const int sq = side * side;
    int x, y;
    if (t < 2 * sq) {
        const bool lo = t < sq;
        dz = lo ? -R : R;
        const int u = lo ? t : t - sq;
        y = small_div(u, side, inv_side);
        x = u - y * side;
    } else {
        const int e = side - 1, per = 4 * e;
        const int u = t - 2 * sq;
        const int layer = small_div(u, per, inv_per);
        const int p = u - layer * per;
        dz = -R + 1 + layer;
        if (p < e) { x = p; y = 0; }
        else if (p < 2 * e) { x = e; y = p - e; }
        else if (p < 3 * e) { x = 3 * e - p; y = e; }
        else { x = 0; y = 4 * e - p; }
    }
    dx = x - R;
    dy = y - R;
}

template <int UCAP, int NB>
struct WarpWalk {
    const GatherGrid& G;
    WarpStore<UCAP, NB>& U;
    V3 q;
    float r;
    int k, lane;
    int n;                    // keys in the store
    int qn;                   // queued sub-cells
    unsigned long long T;     // a candidate enters when its key < T
    float lim, lim2;          // distance bound for pruning; squared pre-filter bound
    float bscale;             // NB / (r or g): distance histogram bin of d = min(NB - 1, (int)(d * bscale))
    bool guessed;             // the first ring ran with a density guess of the bound
    bool failed;              // ... and found fewer than k photons within it: walk again without

    __device__ WarpWalk(const GatherGrid& g, WarpStore<UCAP, NB>& u, V3 qq, float rr, int kk, int ln)
        : G(g), U(u), q(qq), r(rr), k(kk), lane(ln), n(0), qn(0), T(~0ull), lim(rr), lim2(rr * rr * 1.000001f),
          bscale((float)NB / rr), guessed(false), failed(false) {
#pragma unroll
        for (int b = 0; b < NB / 32; b++) U.dh[b * 32 + lane] = 0u;
        __syncwarp();
    }

    // back to the empty store and the bound r
    __device__ void reset() {
        n = 0;
        qn = 0;
        T = ~0ull;
        lim = r;
        lim2 = r * r * 1.000001f;
        bscale = (float)NB / r;
        guessed = failed = false;
        __syncwarp();
#pragma unroll
        for (int b = 0; b < NB / 32; b++) U.dh[b * 32 + lane] = 0u;
        __syncwarp();
    }

    // Density guess of the bound before the first ring's photons are scanned:
    // its N photons lie in the 3 x 3 x 3 block of sub-cells of edge sc around
    // the query; spread over a plane through the block (area 9 sc^2) they give
    // about G.guess x k photons within g = 3 sc sqrt(G.guess k / (pi N)).  The
    // guess filters which candidates enter the store, and a ring-1 sub-cell
    // whose padded box lies farther than g is not scanned at all; when fewer
    // than k photons lie within g, the walk starts again with the bound r, so
    // the answer is unchanged.  One lane per ring-1 sub-cell (all 27 in one
    // round): (a, b) its photon range (empty when it is out of reach), gap2 its
    // squared box distance.
    __device__ void guess_ring1(uint32_t a, uint32_t& b, float gap2, float sc, float m) {
        if (!(G.guess > 0.f)) return;
        uint32_t c = b - a;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
        if (c <= (uint32_t)k) return;   // too few photons in the block to gain anything
        const float g = 3.f * sc * sqrtf(G.guess * (float)k / (3.14159265f * (float)c));
        if (g < lim) {
            lim = g;
            lim2 = g * g * 1.000001f;
            guessed = true;
            bscale = (float)NB / g;   // no candidate is stored yet: the histogram spans [0, g] from here on
            const float L = g * m;
            if (gap2 > L * L) b = a;
        }
    }

    __device__ __forceinline__ uint32_t bin_of(float d) const {
        return (uint32_t)min((int)(d * bscale), NB - 1);   // non-decreasing in d
    }

    // The k-th smallest key of the store (n > k).  The distance histogram
    // locates the bin holding it; the keys of that bin (normally a handful)
    // are sorted by one warp, else the radix select runs over the store.
    __device__ unsigned long long kth_key() {
        uint32_t c[NB / 32], sum = 0;
#pragma unroll
        for (int b = 0; b < NB / 32; b++) { c[b] = U.dh[(NB / 32) * lane + b]; sum += c[b]; }
        uint32_t incl = sum;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += y;
        }
        const uint32_t excl = incl - sum;
        const unsigned own = __ballot_sync(0xffffffffu, excl < (uint32_t)k && (uint32_t)k <= incl);
        const int owner = own ? __ffs(own) - 1 : 0;
        uint32_t bin = 0, before = 0, cnt = 0;
        if (lane == owner) {
            uint32_t run = excl;
#pragma unroll
            for (int b = 0; b < NB / 32; b++) {
                if (cnt == 0 && (uint32_t)k <= run + c[b]) { bin = (NB / 32) * lane + b; before = run; cnt = c[b]; }
                run += c[b];
            }
        }
        bin = __shfl_sync(0xffffffffu, bin, owner);
        before = __shfl_sync(0xffffffffu, before, owner);
        cnt = __shfl_sync(0xffffffffu, cnt, owner);
        if (!own || cnt > 32u) return select_kth(U, n, k, lane);
        int got = 0;
        for (int base = 0; base < n; base += 32) {
            const int i = base + lane;
            const unsigned long long kk = i < n ? U.key[i] : ~0ull;
            const bool m = i < n && bin_of(__uint_as_float((uint32_t)(kk >> 32))) == bin;
            const unsigned bm = __ballot_sync(0xffffffffu, m);
            if (m) U.sel[got + __popc(bm & lanemask_lt())] = kk;
            got += __popc(bm);
        }
        __syncwarp();
        // the bin holds a handful of keys (unique): rank each against the
        // others instead of sorting 32 lanes
        const unsigned long long mine = lane < got ? U.sel[lane] : ~0ull;
        __syncwarp();
        int rank = 0;
        for (int j = 0; j < got; j++) rank += shfl_u64(mine, j) < mine ? 1 : 0;
        const unsigned hit = __ballot_sync(0xffffffffu, lane < got && rank == k - (int)before - 1);
        return shfl_u64(mine, __ffs(hit) - 1);
    }

    // Tighten the distance bound from the histogram alone (n > k): the k-th
    // smallest distance lies in the bin where the running count reaches k, so
    // the bin's upper edge (with a margin over the rounding of d * bscale) bounds it.
    __device__ void bound() {
        uint32_t c[NB / 32], sum = 0;
#pragma unroll
        for (int b = 0; b < NB / 32; b++) { c[b] = U.dh[(NB / 32) * lane + b]; sum += c[b]; }
        uint32_t incl = sum;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += y;
        }
        const uint32_t excl = incl - sum;
        const unsigned own = __ballot_sync(0xffffffffu, excl < (uint32_t)k && (uint32_t)k <= incl);
        if (!own) return;
        const int owner = __ffs(own) - 1;
        int bin = 0;
        if (lane == owner) {
            uint32_t run = excl;
            bool found = false;
#pragma unroll
            for (int b = 0; b < NB / 32; b++) {
                if (!found && (uint32_t)k <= run + c[b]) { bin = (NB / 32) * lane + b; found = true; }
                run += c[b];
            }
        }
        bin = __shfl_sync(0xffffffffu, bin, owner);
        const float edge = (float)(bin + 1) / bscale * (1.f + 1e-5f);
        if (edge < lim) {
            lim = edge;
            lim2 = lim * lim * 1.000001f;
        }
    }

    // keep the k best keys of the store, tighten the threshold (last: the
    // walk is over, so the histogram need not count the kept keys again)
    __device__ void merge(bool last = false) {
        __syncwarp();
        if (n > k) {
            T = kth_key();
            int w = 0;
            for (int base = 0; base < n; base += 32) {
                int i = base + lane;
                unsigned long long kk = i < n ? U.key[i] : 0ull;
                uint32_t sl = i < n ? U.slot[i] : 0u;
                bool keep = i < n && kk <= T;
                unsigned m = __ballot_sync(0xffffffffu, keep);
                __syncwarp();
                if (keep) {
                    int pos = w + __popc(m & lanemask_lt());
                    U.key[pos] = kk;
                    U.slot[pos] = sl;
                }
                w += __popc(m);
                __syncwarp();
            }
            n = w;
            if (!last) {
                // the histogram counts the store's keys again
#pragma unroll
                for (int b = 0; b < NB / 32; b++) U.dh[b * 32 + lane] = 0u;
                __syncwarp();
                for (int i = lane; i < n; i += 32) atomicAdd(&U.dh[bin_of(__uint_as_float((uint32_t)(U.key[i] >> 32)))], 1u);
            }
        } else if (n == k) {
            T = warp_max_key(U, n, lane);
        }
        if (n == k) {
            lim = fminf(r, __uint_as_float((uint32_t)(T >> 32)));
            lim2 = lim * lim * 1.000001f;
        }
        __syncwarp();
    }

    // test photon slot j (when valid); survivors enter the store
    __device__ __forceinline__ void consider(float4 p, uint32_t j, bool valid) {
        bool ok = false;
        unsigned long long kk = 0ull;
        float d = 0.f;
        if (valid) {
            float dx = p.x - q.x, dy = p.y - q.y, dz = p.z - q.z;
            float s = dx * dx + dy * dy + dz * dz;
            if (s <= lim2) {
                d = sqrtf(s);
                if (d <= r) {
                    kk = ((unsigned long long)__float_as_uint(d) << 32) | __float_as_uint(p.w);
                    ok = kk < T;
                }
            }
        }
        const unsigned m = __ballot_sync(0xffffffffu, ok);
        if (m) {
            if (ok) {
                const int pos = n + __popc(m & lanemask_lt());
                U.key[pos] = kk;
                U.slot[pos] = j;
                atomicAdd(&U.dh[bin_of(d)], 1u);
            }
            n += __popc(m);
            if (n + 32 > UCAP) merge();
        }
    }

    // Scan the photons of queued sub-cells [0, cnt) (cnt <= 32) as one list:
    // lane l takes list entries base + l + 32 i (i < 4), so one round of loads
    // covers 128 photons whichever sub-cells they belong to.
    __device__ void drain(int cnt) {
        constexpr int NL = 1;
        __syncwarp();
        uint32_t a = 0u, c = 0u;
        if (lane < cnt) { a = U.qa[lane]; c = U.qc[lane]; }
        uint32_t incl = c;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += y;
        }
        const uint32_t total = __shfl_sync(0xffffffffu, incl, 31);
        const uint32_t excl = incl - c;
        for (uint32_t base = 0; base < total; base += 32 * NL) {
            uint32_t j[NL];
            bool v[NL];
            float4 p[NL];
#pragma unroll
            for (int u = 0; u < NL; u++) {
                const uint32_t b0 = base + 32 * u, o = b0 + lane;
                // the last queued sub-cell whose first list entry is <= o: the
                // sub-cells that start before this round, plus those starting in
                // it at or before this lane (starts are distinct: queued
                // sub-cells are non-empty)
                const bool valid = lane < cnt;
                const uint32_t starts =
                    __reduce_or_sync(0xffffffffu, valid && excl >= b0 && excl - b0 < 32u ? 1u << (excl - b0) : 0u);
                const int before = __popc(__ballot_sync(0xffffffffu, valid && excl < b0));
                const uint32_t upto = lane == 31 ? 0xffffffffu : (2u << lane) - 1u;
                const int mm = before + __popc(starts & upto) - 1;
                j[u] = __shfl_sync(0xffffffffu, a, mm) + (o - __shfl_sync(0xffffffffu, excl, mm));
                v[u] = o < total;
            }
#pragma unroll
            for (int u = 0; u < NL; u++) p[u] = v[u] ? __ldg(G.gpos + j[u]) : make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
            for (int u = 0; u < NL; u++)
                if (base + 32 * u < total) consider(p[u], j[u], v[u]);
        }
        __syncwarp();
    }

    // append this lane's sub-cell (when ok) to the queue; drain 32 when it holds 32
    __device__ __forceinline__ void enqueue(bool ok, uint32_t a, uint32_t c) {
        const unsigned m = __ballot_sync(0xffffffffu, ok);
        if (ok) {
            const int pos = qn + __popc(m & lanemask_lt());
            U.qa[pos] = a;
            U.qc[pos] = c;
        }
        qn += __popc(m);
        if (qn >= 32) {
            drain(32);
            const int rest = qn - 32;
            uint32_t ra = 0u, rc = 0u;
            if (lane < rest) { ra = U.qa[32 + lane]; rc = U.qc[32 + lane]; }
            __syncwarp();
            if (lane < rest) { U.qa[lane] = ra; U.qc[lane] = rc; }
            __syncwarp();
            qn = rest;
        }
    }

    __device__ __forceinline__ void flush() {
        if (qn > 0) drain(qn);
        qn = 0;
    }

    // Nearest-first walk over the sub-cells of the reference's cube of cells
    // [lo, hi] (global sub-cell coordinates): the query's sub-cell with the
    // shell at Chebyshev distance 1, then, once k candidates are in the store,
    // the remaining sub-cells of the bounding box of the bound's sphere in one
    // pass (box_rest); in sparse regions shells R = 2, 3, ... nearest first.
    // Lanes test 32 sub-cells at a time (box distance against the current
    // bound, non-empty photon range); the survivors are queued and scanned
    // together.  After each shell the distance histogram tightens the bound; a
    // shell whose nearest possible point is farther than the bound ends the walk.
    __device__ void walk(int X0, int Y0, int Z0, int lx, int ly, int lz, int hx, int hy, int hz, bool use_guess) {
        const int S = G.S, sh = __ffs(S) - 1;
        const float sc = G.cell / (float)S, pad = G.cell * 1e-4f;
        const float m = 1.f + 1e-5f;
        const int GX = G.gx * S - 1, GY = G.gy * S - 1, GZ = G.gz * S - 1;
        const uint32_t S3 = (uint32_t)(S * S * S);
        auto key_of = [&](int X, int Y, int Z) -> uint32_t {
            const uint32_t cellid = (uint32_t)((X >> sh) + (Y >> sh) * G.gx + (Z >> sh) * G.gx * G.gy);
            return cellid * S3 + (uint32_t)((X & (S - 1)) + S * ((Y & (S - 1)) + S * (Z & (S - 1))));
        };
        const int Rmax = max(max(max(X0 - lx, hx - X0), max(Y0 - ly, hy - Y0)), max(Z0 - lz, hz - Z0));
        if (Rmax == 0) {   // the query's sub-cell is the whole cube
            const uint32_t key = key_of(X0, Y0, Z0);
            uint32_t a = 0u, b = 0u;
            if (lane == 0) { a = __ldg(G.key_starts + key); b = __ldg(G.key_starts + key + 1); }
            enqueue(lane == 0 && b > a, a, b - a);
            flush();
            return;
        }
        for (int R = 1; R <= Rmax; R++) {
            if ((float)(R - 1) * sc - pad > lim * m) break;
            if (R == 2 && n >= k) {
                // lim now bounds the k-th distance: visit only the sub-cells of
                // its sphere's bounding box outside the 3x3x3 block done
                box_rest(X0, Y0, Z0, lx, ly, lz, hx, hy, hz, sc, pad, m, GX, GY, GZ, S3, sh);
                break;
            }
            const int side = 2 * R + 1;
            const int shell = 2 * side * side + 4 * (side - 1) * (side - 2);
            const int total = shell + (R == 1 ? 1 : 0);   // ring 1 also carries the query's own sub-cell
            const float inv_side = 1.0f / (float)side, inv_per = 1.0f / (float)(4 * (side - 1));
            const float L = lim * m;
            for (int base = 0; base < total; base += 32) {
                const int t = base + lane;
                uint32_t a = 0u, b = 0u;
                float gap2 = 0.f;
                if (t < total) {
                    int dx = 0, dy = 0, dz = 0;
                    if (R == 1) {   // ring 1 with the query's own sub-cell: the 3x3x3 block
                        const int t3 = t / 3, t9 = t3 / 3;
                        dx = t - 3 * t3 - 1;
                        dy = t3 - 3 * t9 - 1;
                        dz = t9 - 1;
                    } else if (t < shell) {
                        shell_member(t, R, side, inv_side, inv_per, dx, dy, dz);
                    }
                    const int X = X0 + dx, Y = Y0 + dy, Z = Z0 + dz;
                    if (X >= lx && X <= hx && Y >= ly && Y <= hy && Z >= lz && Z <= hz) {
                        float ax = axis_gap(q.x, G.mn[0] + X * sc - pad, G.mn[0] + (X + 1) * sc + pad, X == 0, X == GX);
                        float ay = axis_gap(q.y, G.mn[1] + Y * sc - pad, G.mn[1] + (Y + 1) * sc + pad, Y == 0, Y == GY);
                        float az = axis_gap(q.z, G.mn[2] + Z * sc - pad, G.mn[2] + (Z + 1) * sc + pad, Z == 0, Z == GZ);
                        gap2 = ax * ax + ay * ay + az * az;
                        if (gap2 <= L * L) {
                            const uint32_t key = key_of(X, Y, Z);
                            a = __ldg(G.key_starts + key);
                            b = __ldg(G.key_starts + key + 1);
                        }
                    }
                }
                // ring 1 (27 sub-cells) is this one round
                if (R == 1 && use_guess) guess_ring1(a, b, gap2, sc, m);
                enqueue(b > a, a, b - a);
            }
            flush();
            if (R == 1 && guessed && n < k) {
                failed = true;
                return;
            }
            if (n >= k) bound();
        }
        flush();
    }

    // Sub-cells X in [ceil((q - L - pad - mn) / sc) - 1, floor((q + L + pad - mn) / sc)]
    // per axis (the padded boxes that can reach the sphere of radius L = lim m
    // around q), clamped to the cube [lo, hi] (boundary sub-cells with an open
    // side are then included whenever the sphere reaches past them), minus the
    // block |X - X0|, |Y - Y0|, |Z - Z0| <= 1; each tested and queued as in walk().
    __device__ void box_rest(int X0, int Y0, int Z0, int lx, int ly, int lz, int hx, int hy, int hz, float sc,
                             float pad, float m, int GX, int GY, int GZ, uint32_t S3, int sh) {
        const float L = lim * m;
        auto range = [&](float qc, float mn, int lo, int hi, int& b0, int& b1) {
            float f0 = ceilf((qc - L - pad - mn) / sc) - 1.f, f1 = floorf((qc + L + pad - mn) / sc);
            b0 = (int)fminf(fmaxf(f0, (float)lo), (float)hi);
            b1 = (int)fminf(fmaxf(f1, (float)lo), (float)hi);
        };
        int x0, x1, y0, y1, z0, z1;
        range(q.x, G.mn[0], lx, hx, x0, x1);
        range(q.y, G.mn[1], ly, hy, y0, y1);
        range(q.z, G.mn[2], lz, hz, z0, z1);
        if (x0 >= X0 - 1 && x1 <= X0 + 1 && y0 >= Y0 - 1 && y1 <= Y0 + 1 && z0 >= Z0 - 1 && z1 <= Z0 + 1) return;
        const int S = G.S;
        const int nx = x1 - x0 + 1, ny = y1 - y0 + 1, nz = z1 - z0 + 1, nxy = nx * ny;
        const int total = nxy * nz;
        const float inv_nx = 1.0f / (float)nx, inv_nxy = 1.0f / (float)nxy;
        for (int base = 0; base < total; base += 32) {
            const int t = base + lane;
            uint32_t a = 0u, b = 0u;
            if (t < total) {
                const int iz = small_div(t, nxy, inv_nxy), rxy = t - iz * nxy;
                const int iy = small_div(rxy, nx, inv_nx), ix = rxy - iy * nx;
                const int X = x0 + ix, Y = y0 + iy, Z = z0 + iz;
                if (abs(X - X0) > 1 || abs(Y - Y0) > 1 || abs(Z - Z0) > 1) {
                    float ax = axis_gap(q.x, G.mn[0] + X * sc - pad, G.mn[0] + (X + 1) * sc + pad, X == 0, X == GX);
                    float ay = axis_gap(q.y, G.mn[1] + Y * sc - pad, G.mn[1] + (Y + 1) * sc + pad, Y == 0, Y == GY);
                    float az = axis_gap(q.z, G.mn[2] + Z * sc - pad, G.mn[2] + (Z + 1) * sc + pad, Z == 0, Z == GZ);
                    if (ax * ax + ay * ay + az * az <= L * L) {
                        const uint32_t cellid = (uint32_t)((X >> sh) + (Y >> sh) * G.gx + (Z >> sh) * G.gx * G.gy);
                        const uint32_t key =
                            cellid * S3 + (uint32_t)((X & (S - 1)) + S * ((Y & (S - 1)) + S * (Z & (S - 1))));
                        a = __ldg(G.key_starts + key);
                        b = __ldg(G.key_starts + key + 1);
                    }
                }
            }
            enqueue(b > a, a, b - a);
        }
    }
};

// one query (one warp): the k nearest photons within r of q and the estimate
// (UNI: G.pow_uniform is honoured; the batch kernel, whose instance table is
// copied per query, reads the power array instead and keeps its registers)
template <int UCAP, int NB, bool UNI = true>
__device__ __forceinline__ void gather_query(const GatherGrid& G, WarpStore<UCAP, NB>& U, int64_t i, V3 q, V3 nrm,
                                             float r, int k, int require_full, const GatherOut& O, int lane) {
    WarpWalk<UCAP, NB> W(G, U, q, r, k, lane);
    int hx, hy, hz, sx, sy, sz;
    locate(q.x, G.mn[0], G.cell, G.gx, G.S, hx, sx);
    locate(q.y, G.mn[1], G.cell, G.gy, G.S, hy, sy);
    locate(q.z, G.mn[2], G.cell, G.gz, G.S, hz, sz);
    const int S = G.S;
    // the query's own sub-cell first, then shells of sub-cells outwards, within the
    // cube of cells of half width ceil(r / cell) (CudaPhotonMapping/PhotonGrid.cu:257-284)
    const int rc = (int)ceilf(r / G.cell);
    const int x0 = max(0, hx - rc), y0 = max(0, hy - rc), z0 = max(0, hz - rc);
    const int x1 = min(G.gx - 1, hx + rc), y1 = min(G.gy - 1, hy + rc), z1 = min(G.gz - 1, hz + rc);
    for (int pass = 0; pass < 2; pass++) {
        W.walk(hx * S + sx, hy * S + sy, hz * S + sz, x0 * S, y0 * S, z0 * S, x1 * S + S - 1, y1 * S + S - 1,
               z1 * S + S - 1, pass == 0);
        if (!W.failed) break;
        W.reset();
    }
    W.merge(!O.ids);
    const int cnt = W.n;
    // after the merge a full store holds exactly the k best keys, the largest being T
    const unsigned long long kmax = cnt >= k ? W.T : (cnt ? warp_max_key(U, cnt, lane) : 0ull);
    const float rk = cnt ? __uint_as_float((uint32_t)(kmax >> 32)) : 0.f;

    // estimate (Raytracer.cuh:110-138): lanes take entries, then a fixed-order
    // reduction.  The filter's two divisions (by 2 r_k^2 and by its norm) are
    // multiplications by reciprocals taken once per query (the estimate
    // changes by float rounding only); a map of uniform power takes each
    // photon's power from the grid parameters instead of loading it (the same
    // products and sums, so a traced map and the same photons given as a list
    // give the same bits).
    V3 res = v3(0.f, 0.f, 0.f);
    if (cnt > 0 && !(require_full && cnt != k)) {
        const float alpha = 1.818f, beta = 1.953f;
        const float fr = rk * rk;
        const float inv_2fr = 1.f / (2.f * fr);
        const float inv_norm = 1.f / (1.f - expf(-beta));
        const bool uni = UNI && G.pow_uniform;
        const V3 pwu = UNI ? v3(G.pw[0], G.pw[1], G.pw[2]) : v3(0.f, 0.f, 0.f);
        for (int e0 = 0; e0 < cnt; e0 += 64) {
            const int ea = e0 + lane, eb = ea + 32;
            const bool va = ea < cnt, vb = eb < cnt;
            const uint32_t sa = va ? U.slot[ea] : 0u, sb = vb ? U.slot[eb] : 0u;
            V3 pda = v3(0.f, 0.f, 0.f), pdb = pda, pwa = pwu, pwb = pwu;
            if (va) {
                pda = ld3(G.gdir + 3 * (size_t)sa);
                if (!uni) pwa = ld3(G.gpow + 3 * (size_t)sa);
            }
            if (vb) {
                pdb = ld3(G.gdir + 3 * (size_t)sb);
                if (!uni) pwb = ld3(G.gpow + 3 * (size_t)sb);
            }
            if (va && vdot(nrm, vneg(pda)) > 0) {
                const float d = __uint_as_float((uint32_t)(U.key[ea] >> 32));
                const float filter = alpha * (1.f - (1.f - expf(-beta * d * d * inv_2fr)) * inv_norm);
                res = vadd(res, vscale(pwa, filter));
            }
            if (vb && vdot(nrm, vneg(pdb)) > 0) {
                const float d = __uint_as_float((uint32_t)(U.key[eb] >> 32));
                const float filter = alpha * (1.f - (1.f - expf(-beta * d * d * inv_2fr)) * inv_norm);
                res = vadd(res, vscale(pwb, filter));
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            res.x += __shfl_xor_sync(0xffffffffu, res.x, o);
            res.y += __shfl_xor_sync(0xffffffffu, res.y, o);
            res.z += __shfl_xor_sync(0xffffffffu, res.z, o);
        }
        float common = 1.f / (3.14159265358979f * (rk * rk) * 1);
        res = vscale(res, common);
    }
    if (lane == 0) {
        st3(O.rad + 3 * i, res);
        if (O.cnt) O.cnt[i] = cnt;
        if (O.rk) O.rk[i] = rk;
    }
    if (O.ids) {
        // ascending (distance, id): bitonic sort of the store's keys (padded to a power of two)
        int P = 32;
        while (P < cnt) P <<= 1;
        for (int e = cnt + lane; e < P; e += 32) U.key[e] = ~0ull;
        __syncwarp();
        for (int size = 2; size <= P; size <<= 1)
            for (int stride = size >> 1; stride > 0; stride >>= 1) {
                for (int e = lane; e < P; e += 32) {
                    int o = e ^ stride;
                    if (o > e) {
                        unsigned long long a = U.key[e], b = U.key[o];
                        bool ascending = (e & size) == 0;
                        if ((a > b) == ascending) { U.key[e] = b; U.key[o] = a; }
                    }
                }
                __syncwarp();
            }
        for (int e = lane; e < k; e += 32)
            O.ids[i * k + e] = e < cnt ? (uint32_t)(U.key[e] & 0xffffffffull) : 0xffffffffu;
    }
}

__device__ __forceinline__ void gather_zero(int64_t i, int k, const GatherOut& O, int lane) {
    if (lane == 0) {
        st3(O.rad + 3 * i, v3(0.f, 0.f, 0.f));
        if (O.cnt) O.cnt[i] = 0;
        if (O.rk) O.rk[i] = 0.f;
    }
    if (O.ids) for (int e = lane; e < k; e += 32) O.ids[i * k + e] = 0xffffffffu;
}

template <int UCAP>
__global__ void __launch_bounds__(WARPS * 32, 4)
k_gather(GatherGrid G, GatherQueries Q, float r, int k, int require_full, GatherOut O) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t qi = (int64_t)blockIdx.x * WARPS + warp;
    if (qi >= Q.n) return;
    const int64_t i = Q.idx ? (int64_t)Q.idx[qi] : qi;
    WarpStore<UCAP, GATHER_BINS>& U = reinterpret_cast<WarpStore<UCAP, GATHER_BINS>*>(smem_raw)[warp];
    V3 q, nrm;
    bool active = true;
    if (Q.pos3) {
        q = ld3(Q.pos3 + 3 * i);
        nrm = ld3(Q.nrm3 + 3 * i);
    } else {
        float4 a = Q.pos4[i], b = Q.nrm4[i];
        active = (__float_as_uint(b.w) & Q.flag_mask) != 0u;
        q = xyz(a);
        nrm = xyz(b);
    }
    if (!active || k <= 0) {
        gather_zero(i, k, O, lane);
        return;
    }
    gather_query<UCAP, GATHER_BINS>(G, U, i, q, nrm, r, k, require_full, O, lane);
}

// Listed queries, persistent: warps take list positions from *queue until
// min(*n_dev, Q.n) is reached (a device-side count, so no host round trip
// sits between the list's producer and this launch); position qi answers
// record Q.idx[qi].
template <int UCAP>
__global__ void __launch_bounds__(WARPS * 32, 4)
k_gather_listed(GatherGrid G, GatherQueries Q, const unsigned long long* __restrict__ n_dev,
                unsigned long long* __restrict__ queue, float r, int k, GatherOut O) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    WarpStore<UCAP, GATHER_BINS>& U = reinterpret_cast<WarpStore<UCAP, GATHER_BINS>*>(smem_raw)[warp];
    const int64_t n = (int64_t)min(*n_dev, (unsigned long long)Q.n);
    while (true) {
        unsigned long long t = 0;
        if (lane == 0) t = atomicAdd(queue, 1ull);
        const int64_t qi = (int64_t)__shfl_sync(0xffffffffu, t, 0);
        if (qi >= n) break;
        const int64_t i = (int64_t)Q.idx[qi];
        const float4 a = Q.pos4[i], b = Q.nrm4[i];
        if (!((__float_as_uint(b.w) & Q.flag_mask) != 0u) || k <= 0) {
            gather_zero(i, k, O, lane);
            continue;
        }
        gather_query<UCAP, GATHER_BINS>(G, U, i, xyz(a), xyz(b), r, k, 0, O, lane);
        __syncwarp();
    }
}

template <int UCAP>
cudaError_t launch_listed(const GatherGrid& G, const GatherQueries& Q, const unsigned long long* n_dev,
                          unsigned long long* queue, float r, int k, const GatherOut& O, int sm_count,
                          cudaStream_t st) {
    const size_t smem = sizeof(WarpStore<UCAP, GATHER_BINS>) * WARPS;
    cudaError_t e = cudaFuncSetAttribute(k_gather_listed<UCAP>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    int per_sm = 0;
    if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_gather_listed<UCAP>, WARPS * 32, smem)) != cudaSuccess)
        return e;
    const int64_t need = (Q.n + WARPS - 1) / WARPS;
    const unsigned grid = (unsigned)std::min<int64_t>(need, (int64_t)std::max(per_sm, 1) * std::max(sm_count, 1));
    k_gather_listed<UCAP><<<grid, WARPS * 32, smem, st>>>(G, Q, n_dev, queue, r, k, O);
    return cudaGetLastError();
}

__device__ __forceinline__ int find_instance_px(const int64_t* __restrict__ off, int ninst, int64_t g) {
    int lo = 0, hi = ninst - 1;   // last i with off[i] <= g
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(off + mid) <= g) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// Requests of several instances, one persistent work queue: warps take
// MULTI_CHUNK request indices at a time from *queue until *n_req (the eye
// pass's device counter of this class) is reached.  Request q belongs to the
// instance of its pixel (c.w bits, a global pixel index in [px_off[i],
// px_off[i+1])) and is answered with that instance's grid, r and k.  The eye
// pass puts every request in its class's range, so an instance of another
// store class never appears here; the check guards the store size.
constexpr int MULTI_CHUNK = 4;
template <int UCAP, int NW>
__global__ void __launch_bounds__(NW * 32, 32 / NW)
k_gather_multi(const GatherInstDev* __restrict__ tab, const int64_t* __restrict__ px_off, int ninst,
               GatherQueries Q, const float4* __restrict__ rec_c, const unsigned long long* __restrict__ n_req,
               unsigned long long* __restrict__ queue, int cls, GatherOut O) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    WarpStore<UCAP, MULTI_BINS>& U = reinterpret_cast<WarpStore<UCAP, MULTI_BINS>*>(smem_raw)[warp];
    const int64_t n = (int64_t)min(*n_req, (unsigned long long)Q.n);
    // the instance of the last request and its pixel range: consecutive
    // requests mostly belong to one instance (the eye pass writes them in
    // instance order), so the search runs only when the pixel leaves the range
    int inst = -1;
    int64_t px_lo = 0, px_hi = 0;
    while (true) {
        unsigned long long t = 0;
        if (lane == 0) t = atomicAdd(queue, (unsigned long long)MULTI_CHUNK);
        const int64_t q0 = (int64_t)__shfl_sync(0xffffffffu, t, 0);
        if (q0 >= n) break;
        const int64_t q1 = min(q0 + (int64_t)MULTI_CHUNK, n);
        for (int64_t i = q0; i < q1; i++) {
            const int64_t px = (int64_t)__float_as_uint(rec_c[i].w);
            if (px < px_lo || px >= px_hi) {
                inst = find_instance_px(px_off, ninst, px);
                px_lo = __ldg(px_off + inst);
                px_hi = __ldg(px_off + inst + 1);
            }
            const GatherInstDev& T = tab[inst];
            if (T.cls != cls) continue;
            const float4 a = Q.pos4[i], b = Q.nrm4[i];
            if (!((__float_as_uint(b.w) & Q.flag_mask) != 0u) || T.k <= 0) {
                gather_zero(i, T.k, O, lane);
                continue;
            }
            const GatherGrid G = T.G;
            gather_query<UCAP, MULTI_BINS, false>(G, U, i, xyz(a), xyz(b), T.r, T.k, 0, O, lane);
            __syncwarp();
        }
    }
}

template <int UCAP>
cudaError_t launch(const GatherGrid& G, const GatherQueries& Q, float r, int k, int require_full, const GatherOut& O,
                   cudaStream_t st) {
    const size_t smem = sizeof(WarpStore<UCAP, GATHER_BINS>) * WARPS;
    cudaError_t e = cudaFuncSetAttribute(k_gather<UCAP>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    unsigned blocks = (unsigned)((Q.n + WARPS - 1) / WARPS);
    k_gather<UCAP><<<blocks, WARPS * 32, smem, st>>>(G, Q, r, k, require_full, O);
    return cudaGetLastError();
}

}  // namespace

template <int UCAP, int NW>
cudaError_t launch_multi(const GatherInstDev* tab, const int64_t* px_off, int ninst, const GatherQueries& Q,
                         const float4* rec_c, const unsigned long long* n_req, unsigned long long* queue, int cls,
                         const GatherOut& O, int sm_count, cudaStream_t st) {
    const size_t smem = sizeof(WarpStore<UCAP, MULTI_BINS>) * NW;
    cudaError_t e = cudaFuncSetAttribute(k_gather_multi<UCAP, NW>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    int per_sm = 0;
    if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_gather_multi<UCAP, NW>, NW * 32, smem)) != cudaSuccess)
        return e;
    k_gather_multi<UCAP, NW><<<(unsigned)(std::max(per_sm, 1) * sm_count), NW * 32, smem, st>>>(
        tab, px_off, ninst, Q, rec_c, n_req, queue, cls, O);
    return cudaGetLastError();
}

cudaError_t gather_multi(const GatherInstDev* tab, const int64_t* px_off, int ninst, const GatherQueries& Q,
                         const float4* rec_c, const unsigned long long* n_req, int64_t split,
                         unsigned long long* queues, const GatherOut& O, int warps, int sm_count, cudaStream_t st) {
    if (Q.n <= 0) return cudaSuccess;
    if (split < 0 || split > Q.n || O.ids || O.cnt || O.rk || Q.idx) return cudaErrorInvalidValue;
    cudaError_t e = cudaMemsetAsync(queues, 0, 16, st);
    if (e != cudaSuccess) return e;
    // class 0: [0, split); class 1: the records from split on, indexed from 0
    GatherQueries Q0 = Q, Q1 = Q;
    Q0.n = split;
    Q1.n = Q.n - split;
    Q1.pos4 = Q.pos4 + split;
    Q1.nrm4 = Q.nrm4 + split;
    GatherOut O1 = O;
    O1.rad = O.rad + 3 * split;
    const float4* c1 = rec_c + split;
    if (warps == 4) {
        if (Q0.n > 0 &&
            (e = launch_multi<256, 4>(tab, px_off, ninst, Q0, rec_c, n_req, queues, 0, O, sm_count, st)) != cudaSuccess)
            return e;
        if (Q1.n > 0) e = launch_multi<512, 4>(tab, px_off, ninst, Q1, c1, n_req + 1, queues + 1, 1, O1, sm_count, st);
        return e;
    }
    if (Q0.n > 0 &&
        (e = launch_multi<256, 8>(tab, px_off, ninst, Q0, rec_c, n_req, queues, 0, O, sm_count, st)) != cudaSuccess)
        return e;
    if (Q1.n > 0) e = launch_multi<512, 8>(tab, px_off, ninst, Q1, c1, n_req + 1, queues + 1, 1, O1, sm_count, st);
    return e;
}

int gather_class(int k) { return k <= 96 ? 0 : 1; }

cudaError_t gather_listed(const GatherGrid& G, const GatherQueries& Q, const unsigned long long* n_dev,
                          unsigned long long* queue, float r, int k, const GatherOut& O, int sm_count,
                          cudaStream_t st) {
    if (Q.n <= 0) return cudaSuccess;
    if (!Q.idx || !Q.pos4 || !Q.nrm4) return cudaErrorInvalidValue;
    cudaError_t e = cudaMemsetAsync(queue, 0, 8, st);
    if (e != cudaSuccess) return e;
    if (k <= 96) return launch_listed<256>(G, Q, n_dev, queue, r, k, O, sm_count, st);
    if (k <= 256) return launch_listed<512>(G, Q, n_dev, queue, r, k, O, sm_count, st);
    return cudaErrorInvalidValue;
}

cudaError_t gather(const GatherGrid& G, const GatherQueries& Q, float r, int k, int require_full,
                   const GatherOut& O, unsigned* status, cudaStream_t st) {
    (void)status;
    if (Q.n <= 0) return cudaSuccess;
    if (k <= 96) return launch<256>(G, Q, r, k, require_full, O, st);
    if (k <= 256) return launch<512>(G, Q, r, k, require_full, O, st);
    return cudaErrorInvalidValue;
}

}  // namespace pm
