// The fused simulation step for sm_100a.
//
// One launch advances every network in the engine by one cycle. Its blocks
// first deliver the spikes of cycles t-1 .. t-D into the input buffer of cycle
// t+1, then run the LIF_brian update of cycle t in chunks of neurons taken from
// a per-cycle counter (reads the synaptic input summed during the previous
// launch, writes the new state, appends fired ids to this cycle's ring slot with
// one atomic per block pass and stores each warp's ballot as a fired-bitmap
// word). Blocks that finish delivering early take most of the update, so the
// bandwidth-bound update fills the tail of the delivery.
//
// The two halves touch disjoint data (the input accumulators are double
// buffered by cycle parity, the fire ring has D+2 slots), so they need no
// barrier between them; the kernel boundary orders consecutive cycles.
// The cycle counter lives on the device and is advanced by the last block to
// finish, so the same launch can be replayed from a CUDA graph with no host
// involvement.
//
// Reference semantics (BSim, paths relative to its root):
//   neuron update  LIFENeuron::update  src/neuron/lif/LIFENeuron.cpp:114-160
//                  (GPU: find_life_neuron + update_life_neuron, src/neuron/lif/lif.cu:9-162)
//   delivery       update_dense_static_hit, src/synapse/static/static.cu:59-96:
//                  at cycle t, ring slot t-d feeds the synapses of delay d
//   ring advance   update_time, src/gpu_utils/runtime.cu:81-92
#include <cuda_runtime.h>
#include <stdint.h>

#include "engine.h"

namespace bsim {

// Synapse rows are read once per spike: stream them past L1 and mark them
// evict-first in L2 (ld.global.cs) so the accumulators stay L2-resident.
static __device__ __forceinline__ uint4 ld_stream16(const uint4 *p) { return __ldcs(p); }
static __device__ __forceinline__ uint2 ld_stream8(const uint2 *p) { return __ldcs(p); }

static __device__ __forceinline__ void red_add_u64(unsigned long long *p, unsigned long long v)
{
    asm volatile("red.global.add.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

// Device error flag: the first error code raised stays (BSIM_DEVERR_*). Every
// later launch on the same flag returns at once, so the host reads the code
// (BSIM_ERR_DEVICE) and no further cycle runs on inconsistent data.
static __device__ __forceinline__ void raise_error(const StepArgs &a, int code) { atomicCAS(a.err, 0, code); }

// ---------------------------------------------------------------------------
// Input-drive neurons (drive.h): Constant_spikes per update_constant_neuron
// (src/neuron/constant/constant.cu:18-22), Poisson_spikes per update_poisson_neuron
// and reset_poisson_neuron (src/neuron/poisson/poisson.cu:29-31, 9-15). Both
// ignore their synaptic input, as their recv() does.
// ---------------------------------------------------------------------------
static __device__ __forceinline__ void drive_update(const StepArgs &a, int kind, int64_t j, int t,
                                                 const ClassParams *c, float4 &st, bool &fired)
{
    if (kind == BSIM_NEURON_CONSTANT) {
        const int cnt = __float_as_int(st.w);
        if (t < __float_as_int(st.z) && __fmul_rn((float)(t - __float_as_int(st.y)), st.x) > (float)cnt) {
            fired = true;
            st.w = __int_as_float(cnt + 1);
        }
    } else {
        const int fc = __float_as_int(st.y);
        if (t == fc && t <= __float_as_int(st.z)) {
            fired = true;
            const uint64_t key = poisson_key(a.input_seed, j - __ldg(&c->id_base), fc);
            const long long nxt = (long long)fc + 1 + poisson_draw(key, st.x, a.vtmp[j], a.ptab) +
                                  __float_as_int(st.w);
            st.y = __int_as_float(nxt > 2147483647LL ? 2147483647 : (int)nxt);
        }
    }
}

// ---------------------------------------------------------------------------
// Phase A: LIF_brian update of a grid-stride share of the neurons.
// Arithmetic follows LIFENeuron::update term by term with every product and
// sum rounded on its own (no FMA contraction), as the reference's x86 build
// evaluates it:  v = ((Cm*v + v_tmp) + i_E*C_E) + i_I*C_I.
// ---------------------------------------------------------------------------
// Fired ids are appended to the cycle's ring slot with one global atomic per
// block and pass: warps publish their ballot counts, warp 0 scans them and
// reserves the block's range (a single counter per cycle would otherwise take
// one same-address atomic per warp).
template <int ACC>
static __device__ __forceinline__ void lif_phase(const StepArgs &a, unsigned long long t, int p, int cur,
                                                 int *s_wcnt)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    // the cycle's chunk counter: the upper half of the ticket word (reset by the last block)
    unsigned *chunk_ctr = a.ticket + 1;
    __shared__ long long s_chunk[2];  // this pass's chunk and the next one's (taken during the pass)
    int32_t *slot_ids = a.ring + (int64_t)cur * a.cap;
    uint32_t *bm = a.bitmap + (int64_t)cur * a.W;
    int32_t *hist = a.pop_hist ? a.pop_hist + (int64_t)(t % (unsigned long long)a.hist_len) * a.n_pops : nullptr;
    const float *vtmp = (a.drive_half > 0 && ((t / (unsigned long long)a.drive_half) & 1ull)) ? a.vtmp_alt : a.vtmp;
    // state trace of this cycle: the row, or -1
    long long tr_k = -1, tr_first = 0, tr_count = 0, tr_steps = 0;
    if (a.trace) {
        const TraceCtl tc = *a.trace_ctl;
        const long long k = (long long)t - tc.t0;
        if (k >= 0 && k < tc.steps) {
            tr_k = k;
            tr_first = tc.first;
            tr_count = tc.count;
            tr_steps = tc.steps;
        }
    }
    int buf = 0;  // s_wcnt is double-buffered by pass, so a pass needs no closing barrier
    int cb = 0;
    if (threadIdx.x == 0) s_chunk[0] = (long long)atomicAdd(chunk_ctr, (unsigned)blockDim.x);
    __syncthreads();
    for (;;) {
        // one pass of blockDim.x neurons per chunk; the next chunk is taken while this one
        // runs (its slot is read only after this pass's two barriers, and this slot is
        // written again only in the next pass, after every thread has read it)
        const int64_t bbase = s_chunk[cb];
        if (bbase >= a.N) break;
        if (threadIdx.x == 0) s_chunk[cb ^ 1] = (long long)atomicAdd(chunk_ctr, (unsigned)blockDim.x);
        cb ^= 1;
        buf ^= 64;
        const int64_t base = bbase + (threadIdx.x & ~31);
        const int64_t j = base + lane;
        bool fired = false;
        int pop = -1;
        if (j < a.N) {
            float4 st = a.state[j];
            int refrac = __float_as_int(st.w);
            const ClassParams *c = a.ctab + a.cls[j];
            float inE, inI;
            if (ACC == BSIM_ACC_EXACT) {
                // the target's input is the (two's-complement) sum over the planes
                longlong2 *acc = reinterpret_cast<longlong2 *>(a.acc) + (int64_t)p * a.n_planes * a.N + j;
                longlong2 q = acc[0];
                for (int k = 1; k < a.n_planes; k++) {
                    const longlong2 r = acc[(int64_t)k * a.N];
                    q.x = (long long)((unsigned long long)q.x + (unsigned long long)r.x);
                    q.y = (long long)((unsigned long long)q.y + (unsigned long long)r.y);
                }
                if (a.acc_clear)
                    for (int k = 0; k < a.n_planes; k++) acc[(int64_t)k * a.N] = make_longlong2(0, 0);
                const float sd = __ldg(&c->scale_down);
                inE = __fmul_rn(__ll2float_rn(q.x), sd);
                inI = __fmul_rn(__ll2float_rn(q.y), sd);
            } else {
                float2 q = reinterpret_cast<const float2 *>(a.acc)[(int64_t)p * a.N + j];
                inE = q.x;
                inI = q.y;
            }
            const int kind = __ldg(&c->kind);
            if (kind == BSIM_NEURON_LIF) {
                if (refrac > 0) {
                    refrac -= 1;  // input of this cycle is dropped
                } else {
                    const float Cm = __ldg(&c->Cm), C_E = __ldg(&c->C_E), C_I = __ldg(&c->C_I);
                    float v = __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(Cm, st.x), vtmp[j]), __fmul_rn(st.y, C_E)),
                                        __fmul_rn(st.z, C_I));
                    float iE = __fmul_rn(__ldg(&c->CE), st.y);
                    float iI = __fmul_rn(__ldg(&c->CI), st.z);
                    if (v >= __ldg(&c->v_thresh)) {
                        fired = true;
                        refrac = __ldg(&c->refrac_time) - 1;
                        v = __ldg(&c->v_reset);
                    } else {
                        iE = __fadd_rn(iE, inE);
                        iI = __fadd_rn(iI, inI);
                    }
                    st.x = v;
                    st.y = iE;
                    st.z = iI;
                }
                st.w = __int_as_float(refrac);
            } else {
                drive_update(a, kind, j, (int)t, c, st, fired);  // input is dropped (recv returns 0)
            }
            a.state[j] = st;
            if (tr_k >= 0 && j >= tr_first && j < tr_first + tr_count) {
                const int64_t plane = tr_steps * tr_count;
                float *row = a.trace + tr_k * tr_count + (j - tr_first);
                row[0] = st.x;
                row[plane] = st.y;
                row[2 * plane] = st.z;
                row[3 * plane] = inE;
                row[4 * plane] = inI;
            }
            if (hist) pop = __ldg(&c->pop);
        }
        const unsigned mask = __ballot_sync(0xffffffffu, fired);
        if (lane == 0 && base < a.N) bm[base >> 5] = mask;
        if (lane == 0) s_wcnt[buf + warp] = __popc(mask);
        __syncthreads();
        if (warp == 0) {
            int c = lane < nwarps ? s_wcnt[buf + lane] : 0;
            const int own = c;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int nb = __shfl_up_sync(0xffffffffu, c, o);
                if (lane >= o) c += nb;
            }
            const int total = __shfl_sync(0xffffffffu, c, 31);
            int at = 0;
            if (lane == 0 && total) at = atomicAdd(&a.ring_cnt[cur], total);
            at = __shfl_sync(0xffffffffu, at, 0);
            if (lane < nwarps) s_wcnt[buf + 32 + lane] = at + c - own;  // this warp's first position
        }
        __syncthreads();
        if (mask) {
            if (fired) {
                slot_ids[s_wcnt[buf + 32 + warp] + __popc(mask & ((1u << lane) - 1u))] = (int32_t)j;
                atomicAdd(&a.fire_count[j], 1);  // a reduction: nothing waits for the old count
            }
            if (hist) {
                // one atomic per (warp, population) with spikes
                const unsigned same = __match_any_sync(0xffffffffu, fired ? pop : -1);
                if (fired && lane == __ffs(same) - 1) atomicAdd(&hist[pop], __popc(same));
            }
        }
        // no barrier here: the next pass writes the other half of s_wcnt, and the pass
        // after it is ordered by the next pass's barriers
    }
}

// ---------------------------------------------------------------------------
// Phase B, push: one warp per (spike, delay) segment of the source-ordered
// rows; 16-byte streaming loads of two packed {target, weight} entries per
// lane; exact int64 red.add into the target's E or I accumulator.
// ---------------------------------------------------------------------------
static __device__ __forceinline__ void push_one(const StepArgs &a, unsigned long long *acc, uint32_t tgt,
                                                uint32_t wbits, float sc)
{
    if ((int64_t)tgt >= a.N) {  // a target outside the network: flag it, touch nothing
        raise_error(a, BSIM_DEVERR_TARGET);
        return;
    }
    const float w = __int_as_float(wbits);
    const long long q = __float2ll_rn(__fmul_rn(w, sc));
    red_add_u64(acc + 2 * (int64_t)tgt + (w >= 0.0f ? 0 : 1), (unsigned long long)q);
}

// (spike, delay) segments whose metadata one warp resolves at once
#ifndef PUSH_CHUNK
#define PUSH_CHUNK 8
#endif
// resident blocks of STEP_MAX_THREADS threads the step kernel is compiled for
// (together they set its register budget: 65,536 / (2 x 512) = 64 per thread)
#ifndef STEP_MAX_THREADS
#define STEP_MAX_THREADS 512
#endif
#ifndef STEP_MIN_BLOCKS
#define STEP_MIN_BLOCKS 2
#endif
#define MAX_WARPS 16

struct PushSeg {
    long long incl;  // inclusive prefix of the chunk's pair counts
    int64_t p0;      // first entry of the segment's first 16-byte pair
    float sc;        // 2^qexp of the segment's network
};

// s_cum[d] = spikes of cycles t-1 .. t-d (the push work items of delays 1..d).
// Run by warp 0 before the LIF phase, so its loads overlap the neuron update;
// the caller's __syncthreads publishes it.
static __device__ __forceinline__ void delay_window_prefix(const StepArgs &a, unsigned long long t, long long *s_cum)
{
    const int lane = threadIdx.x & 31;
    const int D = a.D;
    long long run = 0;
    for (int d0 = 1; d0 <= D; d0 += 32) {
        const int d = d0 + lane;
        long long c = 0;
        if (d <= D && (long long)t - d >= 0) c = a.ring_cnt[(t - d) % (unsigned long long)a.R];
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            long long nb = __shfl_up_sync(0xffffffffu, c, o);
            if (lane >= o) c += nb;
        }
        if (d <= D) s_cum[d] = run + c;
        run += __shfl_sync(0xffffffffu, c, 31);
    }
    if (lane == 0) s_cum[0] = 0;
}

static __device__ __forceinline__ unsigned long long push_phase(const StepArgs &a, unsigned long long t, int pw,
                                                                const long long *s_cum, PushSeg *s_seg)
{
    const int lane = threadIdx.x & 31;
    const int D = a.D;
    const long long total = s_cum[D];
    unsigned long long ev = 0;
    unsigned long long *acc = reinterpret_cast<unsigned long long *>(a.acc) + 2 * (int64_t)pw * a.n_planes * a.N;
    const long long n_warps = ((long long)gridDim.x * blockDim.x) >> 5;
    // Segments per warp chunk: PUSH_CHUNK when there are enough for every warp, fewer
    // (down to one) when a cycle has few spikes with long rows, so that more warps
    // share the rows. Chunks go to warps block-interleaved (chunk c to warp c / grid of
    // block c % grid), so a cycle with few chunks still spreads over every SM.
    int pc = PUSH_CHUNK;
    while (pc > 1 && total < (long long)pc * n_warps) pc >>= 1;
    const long long n_chunks = (total + pc - 1) / pc;
    const long long warp_lin = (long long)(threadIdx.x >> 5) * gridDim.x + blockIdx.x;
    for (long long ch = warp_lin; ch < n_chunks; ch += n_warps) {
        // Lanes 0..PUSH_CHUNK-1 each resolve one (spike, delay) segment: its row
        // [r0, r1), split into an odd head entry, 16-byte pairs [p0, p0 + 2*np)
        // and an odd tail entry.
        int64_t r0 = 0, r1 = 0;
        float sc = 0.0f;
        const long long item = ch * pc + lane;
        if (lane < pc && item < total) {
            int lo = 1, hi = D;
            while (lo < hi) {
                const int mid = (lo + hi) >> 1;
                if (s_cum[mid] > item) hi = mid;
                else lo = mid + 1;
            }
            const int d = lo;
            const int slot = (int)((t - d) % (unsigned long long)a.R);
            const int32_t s = a.ring[(int64_t)slot * a.cap + (item - s_cum[d - 1])];
            r0 = a.row_off[(int64_t)s * D + d - 1];
            r1 = a.row_off[(int64_t)s * D + d];
            if (r1 < r0) {  // row offsets not ascending: flag it, skip the row
                raise_error(a, BSIM_DEVERR_ROW);
                r1 = r0;
            }
            sc = __ldg(&a.ctab[a.cls[s]].scale_up);
            ev += (unsigned long long)(r1 - r0);
        }
        const int64_t p0 = (r0 & 1) && r0 < r1 ? r0 + 1 : r0;  // first entry of the first pair
        const long long np = (r1 - p0) >> 1;
        const bool head = p0 != r0, tail = ((r1 - p0) & 1) != 0;
        // inclusive prefix of pair counts over the chunk's segments
        long long incl = np;
#pragma unroll
        for (int o = 1; o < PUSH_CHUNK; o <<= 1) {
            const long long nb = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += nb;
        }
        // the chunk's segment table, in this warp's slice of shared memory
        PushSeg *seg = s_seg + (threadIdx.x >> 5) * PUSH_CHUNK;
        __syncwarp();
        if (lane < PUSH_CHUNK) {
            seg[lane].incl = incl;
            seg[lane].p0 = p0;
            seg[lane].sc = sc;
        }
        __syncwarp();
        const long long total_pairs = __shfl_sync(0xffffffffu, incl, PUSH_CHUNK - 1);
        // head / tail single entries: lane L handles segment L>>1, head if L even
        {
            const int k = lane >> 1;
            const bool want_head = (lane & 1) == 0;
            const bool hk = __shfl_sync(0xffffffffu, head, k & (PUSH_CHUNK - 1));
            const bool tk = __shfl_sync(0xffffffffu, tail, k & (PUSH_CHUNK - 1));
            const int64_t rk0 = __shfl_sync(0xffffffffu, r0, k & (PUSH_CHUNK - 1));
            const int64_t rk1 = __shfl_sync(0xffffffffu, r1, k & (PUSH_CHUNK - 1));
            const float sk = __shfl_sync(0xffffffffu, sc, k & (PUSH_CHUNK - 1));
            if (k < PUSH_CHUNK && ((want_head && hk) || (!want_head && tk))) {
                const uint2 x = ld_stream8(a.syn + (want_head ? rk0 : rk1 - 1));
                push_one(a, acc, x.x, x.y, sk);
            }
        }
        // the pairs of all segments as one flat range, four loads in flight per lane
        // each chunk walks its range from its own starting point (wrapping around), so that
        // chunks whose rows hit the same targets (a population's sources in a dense
        // projection) do not add into the same addresses in lockstep
        const long long rot = total_pairs > 0 ? (long long)((unsigned long long)(ch * 40503ll) % total_pairs) : 0;
        for (long long pb = 0; pb < total_pairs; pb += 4 * 32) {
            uint4 x[4];
            float xs[4];
            bool ok[4];
#pragma unroll
            for (int u = 0; u < 4; u++) {
                const long long q = pb + u * 32 + lane;
                ok[u] = q < total_pairs;
                const long long p = q + rot < total_pairs ? q + rot : q + rot - total_pairs;
                int k = 0;
                while (k < PUSH_CHUNK - 1 && p >= seg[k].incl) k++;
                const long long excl = k == 0 ? 0 : seg[k - 1].incl;
                xs[u] = seg[k].sc;
                if (ok[u]) x[u] = ld_stream16(reinterpret_cast<const uint4 *>(a.syn + seg[k].p0) + (p - excl));
            }
#pragma unroll
            for (int u = 0; u < 4; u++) {
                if (ok[u]) {
                    push_one(a, acc, x[u].x, x[u].y, xs[u]);
                    push_one(a, acc, x[u].z, x[u].w, xs[u]);
                }
            }
        }
    }
    return ev;
}

// ---------------------------------------------------------------------------
// Phase B, pull: one warp per target over its target-ordered row (creation
// order), testing each source's bit in the fired bitmap of cycle t - delay.
// EXACT: int64 fixed-point partial sums, warp-reduced (order-free).
// ORDERED: the active weights of each 32-entry chunk are added one by one in
// row order with warp shuffles, so the fp32 sum is formed in exactly the order
// of the reference's loop over pSynapses.
// ---------------------------------------------------------------------------
template <int ACC>
static __device__ __forceinline__ unsigned long long pull_phase(const StepArgs &a, unsigned long long t, int pw)
{
    const int lane = threadIdx.x & 31;
    const long long n_warps = ((long long)gridDim.x * blockDim.x) >> 5;
    unsigned long long ev = 0;
    for (long long j = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; j < a.N; j += n_warps) {
        const int64_t c0 = a.col_off[j], c1 = a.col_off[j + 1];
        const float sc = (ACC == BSIM_ACC_EXACT) ? __ldg(&a.ctab[a.cls[j]].scale_up) : 0.0f;
        long long sE = 0, sI = 0;
        float fE = 0.0f, fI = 0.0f;
        for (int64_t k0 = c0; k0 < c1; k0 += 32) {
            const int64_t e = k0 + lane;
            bool act = false;
            float w = 0.0f;
            if (e < c1) {
                const uint32_t s = __ldcs(a.csc_src + e);
                const int d = (int)__ldcs(a.csc_d + e) + 1;
                w = __ldcs(a.csc_w + e);
                if ((long long)t - d >= 0) {
                    const int slot = (int)((t - d) % (unsigned long long)a.R);
                    act = (a.bitmap[(int64_t)slot * a.W + (s >> 5)] >> (s & 31)) & 1u;
                }
            }
            unsigned m = __ballot_sync(0xffffffffu, act);
            ev += __popc(m);
            if (ACC == BSIM_ACC_EXACT) {
                if (act) {
                    const long long q = __float2ll_rn(__fmul_rn(w, sc));
                    if (w >= 0.0f) sE += q;
                    else sI += q;
                }
            } else {
                while (m) {
                    const int b = __ffs(m) - 1;
                    const float wb = __shfl_sync(0xffffffffu, w, b);
                    if (wb >= 0.0f) fE = __fadd_rn(fE, wb);
                    else fI = __fadd_rn(fI, wb);
                    m &= m - 1;
                }
            }
        }
        if (ACC == BSIM_ACC_EXACT) {
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                sE += __shfl_xor_sync(0xffffffffu, sE, o);
                sI += __shfl_xor_sync(0xffffffffu, sI, o);
            }
            if (lane == 0)
                reinterpret_cast<longlong2 *>(a.acc)[(int64_t)pw * a.n_planes * a.N + j] = make_longlong2(sE, sI);
        } else {
            if (lane == 0) reinterpret_cast<float2 *>(a.acc)[(int64_t)pw * a.N + j] = make_float2(fE, fI);
        }
    }
    return lane == 0 ? ev : 0ull;
}

// ---------------------------------------------------------------------------
// Phase B, tiled: the exact E and I sums of a tile of target neurons are formed
// in shared memory, so no per-event global atomic is issued. Tiles follow
// population boundaries and hold up to a few thousand targets (16 bytes of
// counters each), so each source's row into a tile stays a long segment. A
// tile's work units are cut into parts; blocks take parts from a per-cycle queue
// (largest first) and, once it is empty, help the parts with the most work
// left. The first block to finish a piece of a tile stores its sums into the
// tile's accumulator plane; the others add theirs after that store.
//
// The tile's synapses are grouped by (source, delay) and its sources form runs
// of consecutive ids. A work unit is (run, delay d, 32-source chunk): one lane
// reads the chunk's word of the fired bitmap of cycle t-d. Each fired
// (source, delay) names one segment of 8-byte entries ({target offset in the
// tile, weight bits}), padded to an even length from an even start; a warp
// gathers up to TILE_SEGS segments and streams them as one flat range of
// 16-byte entry pairs, each lane advancing its own segment cursor.
//
// Exact int64 sums with 32-bit shared atomics: the low word of the fixed-point
// value is added with an atomic that returns the old word, and the high word
// plus the carry out of the low word with a second one. After all additions the
// (high, low) pair is the exact two's-complement sum (additions commute, and
// every carry is counted once); the fixed-point exponent keeps every sum below
// 2^61, so the high word cannot overflow.
// ---------------------------------------------------------------------------
#ifndef TILE_HELP_MIN
#define TILE_HELP_MIN 64  // units a part must have left per helping block for another block to join
#endif
#ifndef TILE_WAIT_SPINS
#define TILE_WAIT_SPINS (1u << 22)  // ~0.3 s of 64 ns sleeps: far beyond any store phase
#endif
#ifndef TILE_SEGS
#define TILE_SEGS 64  // fired segments a warp lists per round
#endif
static_assert(TILE_SEGS >= 32 && TILE_SEGS <= 64, "a round's segment prefix covers two entries per lane");
#ifndef TILE_CHUNK_PAIRS
#define TILE_CHUNK_PAIRS 512  // entry pairs a chunk of units should list (from the previous cycle's rate)
#endif
#ifndef TILE_MIN_CHUNK
#define TILE_MIN_CHUNK 8ll  // units per chunk at least
#endif
#ifndef TILE_INFLIGHT
#define TILE_INFLIGHT 4  // 16-byte entry pairs per lane loaded before they are added
#endif

// Counters are [4][tile]: E low, E high, I low, I high words (word-major, so
// lanes adding into scattered targets spread over all shared-memory banks).
static __device__ __forceinline__ void carry_add(unsigned *lo, int T, long long v)
{
    const unsigned long long u = (unsigned long long)v;
    const unsigned l = (unsigned)u, h = (unsigned)(u >> 32);
    const unsigned old = atomicAdd(lo, l);
    atomicAdd(lo + T, h + (old + l < old ? 1u : 0u));
}

// Two entries at once: both low words first, so the second atomic's latency
// overlaps the first's (a returned value is waited for only where it is used).
static __device__ __forceinline__ void carry_add2(unsigned *lo0, long long v0, unsigned *lo1, long long v1, int T)
{
    const unsigned long long u0 = (unsigned long long)v0, u1 = (unsigned long long)v1;
    const unsigned l0 = (unsigned)u0, l1 = (unsigned)u1;
    const unsigned o0 = atomicAdd(lo0, l0);
    const unsigned o1 = atomicAdd(lo1, l1);
    atomicAdd(lo0 + T, (unsigned)(u0 >> 32) + (o0 + l0 < o0 ? 1u : 0u));
    atomicAdd(lo1 + T, (unsigned)(u1 >> 32) + (o1 + l1 < o1 ? 1u : 0u));
}

static __device__ __forceinline__ long long carry_sum(const unsigned *lo, int T)
{
    return (long long)(((unsigned long long)lo[T] << 32) | (unsigned long long)lo[0]);
}

static __device__ __forceinline__ unsigned long long tile_phase(const StepArgs &a, unsigned long long t, int pw,
                                                                unsigned *s_acc, long long *s_start, int *s_cum,
                                                                int *s_part)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int D = a.D;
    long long *seg_start = s_start + warp * TILE_SEGS;
    int *seg_cum = s_cum + warp * TILE_SEGS;
    unsigned long long ev = 0;
    unsigned long long *s_best = reinterpret_cast<unsigned long long *>(s_part + 2);
    // the counters start at zero once per launch; each part's flush clears what it read,
    // so the next part (any tile size up to tile_max) finds them zero
    for (int i = threadIdx.x; i < 4 * a.tile_max; i += blockDim.x) s_acc[i] = 0u;
    for (;;) {
        if (threadIdx.x == 0) {
            const unsigned q = atomicAdd(a.part_ctr, 1u);
            s_part[0] = q < (unsigned)a.n_parts ? (int)q : -1;
            *s_best = 0ull;
        }
        __syncthreads();
        int pi = s_part[0];
        const bool helper = pi < 0;
        if (helper) {
            // the queue is empty: join the part with the most units left per block already
            // helping it (at least two chunks each), so that helpers spread over the parts
            unsigned long long best = 0ull;
            for (int i = threadIdx.x; i < a.n_parts; i += blockDim.x) {
                const unsigned nx = *reinterpret_cast<volatile unsigned *>(a.part_next + i);
                const unsigned end = (unsigned)a.parts[i].z;
                const unsigned hp = *reinterpret_cast<volatile unsigned *>(a.part_help + i);
                const unsigned left = (nx < end ? end - nx : 0u) / (hp + 1u);
                const unsigned long long key = ((unsigned long long)left << 32) | (unsigned)i;
                best = key > best ? key : best;
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                const unsigned long long other = __shfl_xor_sync(0xffffffffu, best, o);
                best = other > best ? other : best;
            }
            if (lane == 0 && best) atomicMax(s_best, best);
            __syncthreads();
            const unsigned long long b = *s_best;
            pi = (b >> 32) >= (unsigned long long)TILE_HELP_MIN ? (int)(b & 0xffffffffull) : -1;
            if (pi >= 0 && threadIdx.x == 0) atomicAdd(a.part_help + pi, 1u);
        }
        __syncthreads();  // every thread has read s_part / s_best before they are written again
        if (pi < 0) break;
        const int4 part = a.parts[pi];  // {tile, first unit, end unit, part within the tile}
        const int q = part.x, u_end = part.z;
        const int tb = a.tile_beg[q], T = a.tile_beg[q + 1] - tb;
        const float sc = a.tile_scale[q];
        const long long seg0 = a.tile_seg0[q];  // the tile's first entry pair
        const int r0 = a.tile_run_off[q], r1 = a.tile_run_off[q + 1];
        // the warps of every block working on the part take chunks of its units as they become
        // free: 32 units (one per lane), fewer where the part listed many entry pairs per unit in
        // the previous cycle, so that a hot chunk does not hold up the block for long
        unsigned *pairs_cnt = a.part_pairs + (int64_t)(t & 1ull) * a.n_parts + pi;
        const unsigned prev = a.part_pairs[(int64_t)((t & 1ull) ^ 1ull) * a.n_parts + pi];
        const int cs = prev == 0u ? 32
                                  : (int)max(TILE_MIN_CHUNK, min(32ll, (long long)TILE_CHUNK_PAIRS * (u_end - part.y) /
                                                                            (long long)prev));
        unsigned listed = 0;
        for (;;) {
            int ub = 0;
            if (lane == 0) ub = (int)atomicAdd(a.part_next + pi, (unsigned)cs);
            ub = __shfl_sync(0xffffffffu, ub, 0);
            if (ub >= u_end) break;
            const int u = ub + lane;
            unsigned m = 0;
            int64_t kbase = 0;
            int d = 1;
            if (lane < cs && u < u_end) {
                int r = r0;
                while (r + 1 < r1 && a.run_unit0[r + 1] <= u) r++;
                const int n_r = a.run_n[r], chunks = (n_r + 31) >> 5;
                const int v = u - a.run_unit0[r];
                d = v / chunks + 1;
                const int c = v - (d - 1) * chunks;
                if ((long long)t - d >= 0) {
                    const int64_t s_first = (int64_t)a.run_src0[r] + 32 * c;
                    const int len = min(32, n_r - 32 * c);
                    const uint32_t *bm = a.bitmap + (int64_t)((t - d) % (unsigned long long)a.R) * a.W;
                    const int64_t wi = s_first >> 5;
                    const int sh = (int)(s_first & 31);
                    unsigned bits = bm[wi];
                    if (sh) bits = (bits >> sh) | ((wi + 1 < a.W ? bm[wi + 1] : 0u) << (32 - sh));
                    m = len == 32 ? bits : (bits & ((1u << len) - 1u));
                    kbase = a.run_pair0[r] + 32 * c;
                }
            }
            while (__any_sync(0xffffffffu, m != 0)) {
                // this round: up to TILE_SEGS fired (source, delay) segments of the warp
                const int cnt = __popc(m);
                int incl = cnt;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const int nb = __shfl_up_sync(0xffffffffu, incl, o);
                    if (lane >= o) incl += nb;
                }
                const int excl = incl - cnt;
                const int total = __shfl_sync(0xffffffffu, incl, 31);
                const int take = max(0, min(cnt, TILE_SEGS - excl));
                // the lane's fired segments, two at a time: both offset loads are issued
                // before either is used (more at once costs registers the streaming loop needs)
                for (int i = 0; i < take; i += 2) {
                    const int b0 = __ffs(m) - 1;
                    m &= m - 1;
                    const bool two = i + 1 < take;
                    const int b1 = two ? __ffs(m) - 1 : b0;
                    if (two) m &= m - 1;
                    // in 16-byte units: segments start on an even entry and have even length
                    const uint32_t *p0 = a.pair_seg + (kbase + b0) * (D + 1) + (d - 1);
                    const uint32_t *p1 = a.pair_seg + (kbase + b1) * (D + 1) + (d - 1);
                    const uint32_t x0 = p0[0], y0 = p0[1], x1 = p1[0], y1 = p1[1];
                    seg_start[excl + i] = seg0 + (long long)x0;
                    seg_cum[excl + i] = (int)(y0 - x0);  // length for now
                    if (two) {
                        seg_start[excl + i + 1] = seg0 + (long long)x1;
                        seg_cum[excl + i + 1] = (int)(y1 - x1);
                    }
                }
                __syncwarp();
                const int nseg = min(total, TILE_SEGS);
                // inclusive prefix of the segment lengths (two per lane)
                int c0 = lane < nseg ? seg_cum[lane] : 0;
                int c1 = lane + 32 < nseg ? seg_cum[lane + 32] : 0;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const int n0 = __shfl_up_sync(0xffffffffu, c0, o);
                    const int n1 = __shfl_up_sync(0xffffffffu, c1, o);
                    if (lane >= o) {
                        c0 += n0;
                        c1 += n1;
                    }
                }
                const int half = __shfl_sync(0xffffffffu, c0, 31);
                __syncwarp();
                if (lane < nseg) seg_cum[lane] = c0;
                if (lane + 32 < nseg) seg_cum[lane + 32] = half + c1;
                __syncwarp();
                const int n_pairs = seg_cum[nseg - 1];  // 16-byte entry pairs of the round
                listed += (unsigned)n_pairs;
                const uint4 *ent2 = reinterpret_cast<const uint4 *>(a.ent);
                // this lane's segment cursor (its flat positions only grow): the current
                // segment's end, its first flat position and its first entry pair, in registers
                int j = 0, seg_end = seg_cum[0], seg_first = 0;
                long long seg_base = seg_start[0];
                for (int f0 = 0; f0 < n_pairs; f0 += TILE_INFLIGHT * 32) {
                    uint4 v[TILE_INFLIGHT];
#pragma unroll
                    for (int uu = 0; uu < TILE_INFLIGHT; uu++) {
                        const int f = f0 + uu * 32 + lane;
                        if (f < n_pairs) {
                            while (seg_end <= f) {
                                seg_first = seg_end;
                                j++;
                                seg_end = seg_cum[j];
                                seg_base = seg_start[j];
                            }
                            v[uu] = ld_stream16(ent2 + seg_base + (f - seg_first));
                        }
                    }
#pragma unroll
                    for (int uu = 0; uu < TILE_INFLIGHT; uu++) {
                        if (f0 + uu * 32 + lane < n_pairs) {
                            // the sign routes the input as LIFENeuron::recv does; padding (only
                            // ever the second entry of a pair) is skipped
                            const float w0 = __uint_as_float(v[uu].y), w1 = __uint_as_float(v[uu].w);
                            unsigned *c0 = s_acc + (w0 >= 0.0f ? 0 : 2 * T) + (int)v[uu].x;
                            const long long q0 = __float2ll_rn(__fmul_rn(w0, sc));
                            if (v[uu].z != TILE_PAD) {
                                carry_add2(c0, q0, s_acc + (w1 >= 0.0f ? 0 : 2 * T) + (int)v[uu].z,
                                           __float2ll_rn(__fmul_rn(w1, sc)), T);
                                ev += 2;
                            } else {
                                carry_add(c0, T, q0);
                                ev += 1;
                            }
                        }
                    }
                }
                __syncwarp();
            }
        }
        if (lane == 0 && listed) atomicAdd(pairs_cnt, listed);
        __syncthreads();
        // Flush into the tile's one accumulator plane. The first block to finish a piece of
        // the tile this cycle (an owner or a helper) stores its sums; every other block waits
        // until that store is done and adds its sums with reductions. The first finisher
        // never waits, so the waits always end; they are bounded all the same.
        if (threadIdx.x == 0) {
            const unsigned k = atomicAdd(a.tile_arrive + q, 1u);
            if (k != 0u) {
                const volatile unsigned *done = a.tile_arrive + a.n_tiles + q;
                unsigned spins = 0;
                while (*done == 0u) {
                    if (++spins > TILE_WAIT_SPINS) {
                        raise_error(a, BSIM_DEVERR_TIMEOUT);
                        break;
                    }
                    __nanosleep(64);
                }
                __threadfence();
            }
            s_part[1] = k == 0u;
        }
        __syncthreads();
        if (s_part[1]) {
            longlong2 *g = reinterpret_cast<longlong2 *>(a.acc) + (int64_t)pw * a.N + tb;
            for (int i = threadIdx.x; i < T; i += blockDim.x) {
                g[i] = make_longlong2(carry_sum(s_acc + i, T), carry_sum(s_acc + 2 * T + i, T));
                s_acc[i] = s_acc[T + i] = s_acc[2 * T + i] = s_acc[3 * T + i] = 0u;
            }
            __threadfence();
            __syncthreads();
            if (threadIdx.x == 0) atomicExch(a.tile_arrive + a.n_tiles + q, 1u);
        } else {
            unsigned long long *g = reinterpret_cast<unsigned long long *>(a.acc) + 2 * ((int64_t)pw * a.N + tb);
            for (int i = threadIdx.x; i < T; i += blockDim.x) {
                const long long e = carry_sum(s_acc + i, T), v = carry_sum(s_acc + 2 * T + i, T);
                s_acc[i] = s_acc[T + i] = s_acc[2 * T + i] = s_acc[3 * T + i] = 0u;
                if (e) red_add_u64(g + 2 * i, (unsigned long long)e);
                if (v) red_add_u64(g + 2 * i + 1, (unsigned long long)v);
            }
        }
        // the next part's queue read (two barriers) orders the flush before the counters' reuse
    }
    return ev;
}

// ---------------------------------------------------------------------------
// Firing predictor, inside the step: one warp per population evaluates the MLP
// on the population's rates of cycles t-1..t-8 (complete when cycle t runs) and
// its mean in-degree, predicting cycle t+1. Lane u holds hidden units u and
// u+32; the second layer reads the first layer's units through shuffles. The
// prediction only feeds scheduling (the delivery choice of later cycles).
// ---------------------------------------------------------------------------
static __device__ __forceinline__ void predict_phase(const StepArgs &a, unsigned long long t)
{
    const int lane = threadIdx.x & 31;
    const float *P = a.mlp;
    const float *W1 = P, *b1 = P + BSIM_MLP_HIDDEN * BSIM_MLP_IN, *W2 = b1 + BSIM_MLP_HIDDEN;
    const float *b2 = W2 + BSIM_MLP_HIDDEN * BSIM_MLP_HIDDEN, *W3 = b2 + BSIM_MLP_HIDDEN, *b3 = W3 + BSIM_MLP_HIDDEN;
    const int H = a.hist_len;
    for (int p = ((int)(blockIdx.x * blockDim.x + threadIdx.x)) >> 5; p < a.n_pops;
         p += (int)((gridDim.x * blockDim.x) >> 5)) {
        const float size = (float)a.pop_size[p];
        float x[BSIM_MLP_IN];
#pragma unroll
        for (int k = 0; k < 8; k++) {
            const long long s = (long long)t - 1 - k;
            x[k] = s >= 0 ? (float)a.pop_hist[(int64_t)(s % H) * a.n_pops + p] / size * 10.0f : 0.0f;
        }
        x[8] = a.pop_indeg[p] * 1e-3f;
        float h1a = b1[lane], h1b = b1[lane + 32];
#pragma unroll
        for (int k = 0; k < BSIM_MLP_IN; k++) {
            h1a = fmaf(W1[lane * BSIM_MLP_IN + k], x[k], h1a);
            h1b = fmaf(W1[(lane + 32) * BSIM_MLP_IN + k], x[k], h1b);
        }
        h1a = fmaxf(h1a, 0.0f);
        h1b = fmaxf(h1b, 0.0f);
        float s_a = b2[lane], s_b = b2[lane + 32];
        for (int k = 0; k < 32; k++) {
            const float ha = __shfl_sync(0xffffffffu, h1a, k), hb = __shfl_sync(0xffffffffu, h1b, k);
            s_a = fmaf(W2[lane * BSIM_MLP_HIDDEN + k], ha, s_a);
            s_a = fmaf(W2[lane * BSIM_MLP_HIDDEN + 32 + k], hb, s_a);
            s_b = fmaf(W2[(lane + 32) * BSIM_MLP_HIDDEN + k], ha, s_b);
            s_b = fmaf(W2[(lane + 32) * BSIM_MLP_HIDDEN + 32 + k], hb, s_b);
        }
        float y = W3[lane] * fmaxf(s_a, 0.0f) + W3[lane + 32] * fmaxf(s_b, 0.0f);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) y += __shfl_xor_sync(0xffffffffu, y, o);
        if (lane == 0) {
            const float pred = fmaxf(y + b3[0], 0.0f) * size * 0.1f;
            a.pred_ring[(int64_t)((t + 1) & 3) * a.n_pops + p] = pred;
            atomicAdd(&a.pred_sum[((t + 1) & 3) * 2 + 0], pred);
            atomicAdd(&a.pred_sum[((t + 1) & 3) * 2 + 1], pred * a.pop_outdeg[p]);
            if (t >= 3) {
                // the prediction made two cycles ago for cycle t-1, now complete
                const float actual = (float)a.pop_hist[(int64_t)((t - 1) % H) * a.n_pops + p];
                const float predicted = a.pred_ring[(int64_t)((t - 1) & 3) * a.n_pops + p];
                atomicAdd(&a.pstats->abs_err, (double)fabsf(predicted - actual));
                atomicAdd(&a.pstats->actual, (double)actual);
            }
        }
    }
}

// Spikes of the cycles a step delivers (t-1 .. t-D), from the ring counts; every
// lane of the calling warp gets the sum.
static __device__ __forceinline__ float window_spikes(const StepArgs &a, unsigned long long t)
{
    const int lane = threadIdx.x & 31;
    float c = 0.0f;
    for (int d = 1 + lane; d <= a.D; d += 32)
        if ((long long)t - d >= 0) c += (float)a.ring_cnt[(t - d) % (unsigned long long)a.R];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
    return c;
}

// The delivery mode of cycle t under BSIM_DELIVERY_AUTO: the cost model of each
// mode (fixed ns per cycle + ns per event) on the cycle's work.
//  * exact schedule (no predictor attached): the work is the exact spike count of
//    the delivered window t-1 .. t-D times the mean out-degree over D (each spike's
//    synapses are spread over the D delays);
//  * learned schedule: the work is the predictor's estimate for cycle t-1's spikes
//    times the mean out-degree, or the exact count of cycle t-1 when the prediction
//    for that cycle missed by more than the tolerance (the fallback).
// Every block computes the same choice from the same device words.
static __device__ __forceinline__ int auto_delivery(const StepArgs &a, unsigned long long t)
{
    if (!a.mlp) {
        const float work = window_spikes(a, t) * a.mean_outdeg / (float)a.D;
        const int dm = (a.n_tiles > 0 && a.cost_tile_a + a.cost_tile_b * work < a.cost_push_a + a.cost_push_b * work)
                           ? BSIM_DELIVERY_TILE
                           : BSIM_DELIVERY_PUSH;
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            a.pstats->cycles += 1;
            a.pstats->tile_cycles += dm == BSIM_DELIVERY_TILE ? 1 : 0;
        }
        return dm;
    }
    float ps = 0.0f, pe = 0.0f, as = 0.0f;
    if (t >= 1) {
        const float *slot = a.pred_sum + ((t - 1) & 3) * 2;
        ps = *reinterpret_cast<const volatile float *>(slot);
        pe = *reinterpret_cast<const volatile float *>(slot + 1);
        as = (float)a.ring_cnt[(t - 1) % (unsigned long long)a.R];
    }
    const bool fallback = t < 3 || fabsf(as - ps) > a.pred_tol * fmaxf(ps, 1.0f);
    // events per cycle: the spikes of one cycle times their out-degree is, at steady
    // activity, what one cycle delivers (its D slots each hold 1/D of those events)
    const float work = fallback ? as * a.mean_outdeg : pe;
    const int dm = (a.n_tiles > 0 && a.cost_tile_a + a.cost_tile_b * work < a.cost_push_a + a.cost_push_b * work)
                       ? BSIM_DELIVERY_TILE
                       : BSIM_DELIVERY_PUSH;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        a.pstats->cycles += 1;
        a.pstats->fallbacks += fallback ? 1 : 0;
        a.pstats->tile_cycles += dm == BSIM_DELIVERY_TILE ? 1 : 0;
    }
    return dm;
}

// Copies the complete ring slot of cycle t-1 into the raster recording.
static __device__ __forceinline__ void record_phase(const StepArgs &a, unsigned long long t)
{
    if (!a.rec || t == 0) return;
    RecCtl rc;
    {
        const volatile RecCtl *v = a.rec;
        rc.next = v->next;
        rc.t0 = v->t0;
        rc.steps = v->steps;
        rc.cap = v->cap;
    }
    const long long ts = (long long)t - 1;
    const long long k = ts - rc.t0;
    if (k < 0 || k >= rc.steps || rc.next != ts) return;
    const int slot = (int)(ts % a.R);
    const int64_t n = a.ring_cnt[slot];
    const int64_t base = a.rec_off[k];
    int64_t room = rc.cap - base;
    if (room < 0) room = 0;
    const int64_t ncopy = n < room ? n : room;
    const int32_t *src = a.ring + (int64_t)slot * a.cap;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < ncopy; i += (int64_t)gridDim.x * blockDim.x)
        a.rec_ids[base + i] = src[i];
}

template <int ACC>
__global__ void __launch_bounds__(STEP_MAX_THREADS, STEP_MIN_BLOCKS) step_kernel(const __grid_constant__ StepArgs a)
{
    __shared__ long long s_cum[BSIM_MAX_DELAY + 1];
    __shared__ PushSeg s_seg[MAX_WARPS * PUSH_CHUNK];
    __shared__ int s_wcnt[128];
    __shared__ unsigned long long s_ev;
    __shared__ __align__(8) int s_part[4];  // tiled delivery: the block's part; [2..3] the best part to join
    __shared__ int s_last;
    // tiled delivery: [4][tile] u32 limb counters (one sign), then per-warp segment lists
    extern __shared__ __align__(16) unsigned long long s_dyn[];
    // a raised error flag stops every later cycle (block-uniform test)
    if (__syncthreads_or(threadIdx.x == 0 && *reinterpret_cast<volatile int32_t *>(a.err) != 0)) return;
    const unsigned long long t = *reinterpret_cast<volatile unsigned long long *>(a.step_ctr);
    const int p = (int)(t & 1ull);
    const int cur = (int)(t % (unsigned long long)a.R);
    int dm = a.deliv_sel ? *a.deliv_sel : a.delivery;
    if (dm == BSIM_DELIVERY_AUTO) dm = a.pstats ? auto_delivery(a, t) : BSIM_DELIVERY_PUSH;
    if (dm == BSIM_DELIVERY_TILE && a.n_tiles == 0) dm = BSIM_DELIVERY_PUSH;
    if (a.mlp && blockIdx.x == 0 && threadIdx.x == 32) {
        // slot t+2 is next written by cycle t+1's prediction
        a.pred_sum[((t + 2) & 3) * 2 + 0] = 0.0f;
        a.pred_sum[((t + 2) & 3) * 2 + 1] = 0.0f;
    }
    const bool push = ACC != BSIM_ACC_ORDERED && dm == BSIM_DELIVERY_PUSH;
    const bool tiled = ACC != BSIM_ACC_ORDERED && dm == BSIM_DELIVERY_TILE;
    if (threadIdx.x == 0) s_ev = 0;
    if (push && threadIdx.x < 32) delay_window_prefix(a, t, s_cum);
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        // slot t+1 is neither written (LIF writes slot t) nor read (delivery reads t-1..t-D) now
        a.ring_cnt[(t + 1) % (unsigned long long)a.R] = 0;
    }
    if (a.pop_hist) {
        int32_t *nxt = a.pop_hist + (int64_t)((t + 1) % (unsigned long long)a.hist_len) * a.n_pops;
        for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < a.n_pops; i += gridDim.x * blockDim.x) nxt[i] = 0;
    }
    record_phase(a, t);
    __syncthreads();  // publishes s_cum and s_ev
    unsigned long long ev;
    if (push) {
        ev = push_phase(a, t, p ^ 1, s_cum, s_seg);
    } else if (tiled) {
        long long *starts = reinterpret_cast<long long *>(s_dyn + 2 * a.tile_max);
        int *cums = reinterpret_cast<int *>(starts + (blockDim.x >> 5) * TILE_SEGS);
        ev = tile_phase(a, t, p ^ 1, reinterpret_cast<unsigned *>(s_dyn), starts, cums, s_part);
    } else {
        ev = pull_phase<ACC>(a, t, p ^ 1);
    }
    if (ev) atomicAdd(&s_ev, ev);
    lif_phase<ACC>(a, t, p, cur, s_wcnt);
    if (a.mlp && a.pop_hist) predict_phase(a, t);
    __syncthreads();
    if (threadIdx.x == 0) {
        if (s_ev) atomicAdd(a.events, s_ev);
        __threadfence();
        s_last = atomicAdd(a.ticket, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (s_last) {
        // every other block has finished this cycle: the parts' unit counters and the
        // tiles' finisher counts start over
        if (tiled) {
            for (int i = threadIdx.x; i < a.n_parts; i += blockDim.x) {
                a.part_next[i] = (unsigned)a.parts[i].y;
                a.part_help[i] = 0u;
            }
            for (int i = threadIdx.x; i < 2 * a.n_tiles; i += blockDim.x) a.tile_arrive[i] = 0u;
        }
        // the next cycle counts its listed pairs from zero (whichever delivery this cycle used)
        if (a.part_pairs)
            for (int i = threadIdx.x; i < a.n_parts; i += blockDim.x)
                a.part_pairs[(int64_t)((t + 1ull) & 1ull) * a.n_parts + i] = 0u;
        if (threadIdx.x == 0) {
            // advance the cycle
            if (a.rec && t > 0) {
                RecCtl *rc = a.rec;
                const long long k = (long long)t - 1 - rc->t0;
                if (k >= 0 && k < rc->steps && rc->next == (long long)t - 1) {
                    const int64_t n = a.ring_cnt[(t - 1) % (unsigned long long)a.R];
                    a.rec_off[k + 1] = a.rec_off[k] + n;
                    rc->next = (long long)t;
                }
            }
            *a.ticket = 0u;
            *(a.ticket + 1) = 0u;  // the update's chunk counter
            if (a.part_ctr) *a.part_ctr = 0u;
            *a.step_ctr = t + 1;
            __threadfence();
        }
    }
}

// Records the last completed cycle (run after a batch of steps, before reading the raster).
__global__ void record_flush_kernel(const StepArgs a)
{
    const unsigned long long t = *a.step_ctr;  // first cycle not yet run
    if (t == 0 || !a.rec) return;
    const RecCtl rc = *a.rec;
    const long long ts = (long long)t - 1;
    const long long k = ts - rc.t0;
    if (k < 0 || k >= rc.steps || rc.next != ts) return;
    const int slot = (int)(ts % a.R);
    const int64_t n = a.ring_cnt[slot];
    const int64_t base = a.rec_off[k];
    int64_t room = rc.cap - base;
    if (room < 0) room = 0;
    const int64_t ncopy = n < room ? n : room;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < ncopy; i += (int64_t)gridDim.x * blockDim.x)
        a.rec_ids[base + i] = a.ring[(int64_t)slot * a.cap + i];
    __syncthreads();
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        a.rec_off[k + 1] = base + n;
        a.rec->next = ts + 1;
    }
}

// Dynamic shared memory of the step kernel: the tile accumulators and the
// per-warp segment lists of tiled delivery (0 when no tiles are built).
size_t step_dynamic_smem(const StepArgs &a, int block)
{
    if (a.n_tiles == 0) return 0;
    return (size_t)4 * a.tile_max * sizeof(unsigned) + (size_t)(block / 32) * TILE_SEGS * (sizeof(long long) + sizeof(int));
}

// The attribute belongs to the kernel, not to an engine: it only ever grows,
// so an engine built later with smaller tiles cannot break an earlier one.
cudaError_t step_set_smem(int accumulate, size_t bytes)
{
    static size_t set_bytes[64][2];
    int dev = 0;
    cudaError_t st = cudaGetDevice(&dev);
    if (st != cudaSuccess) return st;
    const int k = accumulate == BSIM_ACC_ORDERED ? 1 : 0;
    if (dev < 0 || dev >= 64 || bytes <= set_bytes[dev][k]) return cudaSuccess;
    if (accumulate == BSIM_ACC_ORDERED)
        st = cudaFuncSetAttribute(step_kernel<BSIM_ACC_ORDERED>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)bytes);
    else
        st = cudaFuncSetAttribute(step_kernel<BSIM_ACC_EXACT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)bytes);
    if (st == cudaSuccess) set_bytes[dev][k] = bytes;
    return st;
}

cudaError_t launch_step(Engine &e)
{
    const size_t smem = step_dynamic_smem(e.a, e.block);
    if (e.opt.accumulate == BSIM_ACC_ORDERED)
        step_kernel<BSIM_ACC_ORDERED><<<e.grid, e.block, smem, e.stream>>>(e.a);
    else
        step_kernel<BSIM_ACC_EXACT><<<e.grid, e.block, smem, e.stream>>>(e.a);
    return cudaGetLastError();
}

// One step on explicit arguments (used by the allocation-free entry point).
cudaError_t launch_step_exact(const StepArgs &a, int grid, int block, cudaStream_t stream)
{
    step_kernel<BSIM_ACC_EXACT><<<grid, block, 0, stream>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_record_flush(Engine &e)
{
    record_flush_kernel<<<1, 256, 0, e.stream>>>(e.a);
    return cudaGetLastError();
}

cudaError_t step_occupancy(int block, int accumulate, int *blocks_per_sm, size_t smem)
{
    if (accumulate == BSIM_ACC_ORDERED)
        return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, step_kernel<BSIM_ACC_ORDERED>, block,
                                                             smem);
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, step_kernel<BSIM_ACC_EXACT>, block, smem);
}

cudaError_t step_occupancy(int block, int accumulate, int *blocks_per_sm)
{
    return step_occupancy(block, accumulate, blocks_per_sm, 0);
}

}  // namespace bsim
