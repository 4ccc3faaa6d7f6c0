// Persistent slice engine: every slice of every wave of a batch in one launch.
//
// The batch's work is a list of items in slice order: for slice s, one row item per block of
// rows of every wave in the slice's active prefix, then one column item per tile of columns of
// the same waves.  The active prefix of slice s is the waves up to the last one with more than s
// slices; a wave inside the prefix whose own slices are done skips its items.  A resident block
// takes the next item from a ticket counter, waits until the item's inputs are complete,
// processes it with the arithmetic of the two slice passes (k_row_tt / k_row, k_col_step_tma),
// and counts it done (j = s - slice0, the slice's index within the launch):
//   row item (s, w):    needs the column items of slice s-1 of wave w  (cols_done[w] >= j * CT)
//   column item (s, w): needs the row items of slice s of wave w        (rows_done[w] >= (j+1) * RB)
// Every dependency of a ticket belongs to an earlier ticket, and a block only waits for tickets
// that were handed to running blocks, so the launch cannot deadlock whatever the number of resident
// blocks.  Each wave's slice counters (rows_done, cols_done) are also its progress: when the column
// items of its last slice are done, the block that finished the last one writes the wave's
// completion time (the device clock).  A dependency wait is bounded (EngineArgs.wait_cycles):
// when it runs out the block records the failure in PassArgs.err and stops; the other blocks stop
// at their next ticket once the error word is set.
//
// The row items read the wave through L2 (another block wrote it during this launch) and the
// column items load their tile by TMA, which also reads through L2; a proxy fence orders the
// block's acquire of the row counter before its tensor-memory-accelerator reads.
#pragma once

namespace msb {

template <int N>
struct EngineLayout {
    using L = FftLayout<N>;
    static constexpr int THREADS = L::ROW_THREADS > L::COL_THREADS ? L::ROW_THREADS : L::COL_THREADS;
    static constexpr int ROWS = THREADS / L::G;                       // rows of one row item
    static constexpr size_t ROW_SCR = (size_t)ROWS * L::SCR_STRIDE_ROW;
    static constexpr size_t COL_SCR = (size_t)L::TC * L::SCR_STRIDE_COL;
    static constexpr size_t SCR = ROW_SCR > COL_SCR ? ROW_SCR : COL_SCR;
    static constexpr int MINB = L::COL_MINB < L::ROW_MINB ? L::COL_MINB : L::ROW_MINB;
    // scratch (also the column tile), one twiddle set, the exp table; 128 bytes of alignment slack
    static constexpr size_t SMEM = sizeof(float2) * (SCR + N + 1024) + 128;
};

__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned* p)
{
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// Thread 0 waits (bounded) until *cnt >= need; the result is shared by the block.  While it
// waits it also watches the launch's error word, so that a failure elsewhere ends the wait early.
__device__ __forceinline__ bool engine_wait(const unsigned* cnt, unsigned need, long long limit, const int* err,
                                            int* flag)
{
    if (threadIdx.x == 0) {
        bool ok = ld_acquire_u32(cnt) >= need;
        if (!ok) {
            const long long t0 = clock64();
            for (;;) {
                __nanosleep(64);
                if (ld_acquire_u32(cnt) >= need) {
                    ok = true;
                    break;
                }
                if ((err && *(const volatile int*)err) || clock64() - t0 > limit) break;
            }
        }
        *flag = ok ? 1 : 0;
    }
    __syncthreads();
    return *flag != 0;
}

// Counts an item done: the block's stores are ordered before the count by the barrier and
// thread 0's fence.
__device__ __forceinline__ unsigned engine_signal(unsigned* cnt)
{
    __syncthreads();
    unsigned old = 0;
    if (threadIdx.x == 0) {
        __threadfence();
        old = atomicAdd(cnt, 1u);
    }
    return old;
}

// MODE is the L2Mode of the wave stores and transmission loads (a template argument: chosen at
// run time it costs registers the transforms need).
template <int N, int ROWOP, int MODE>
__global__ void __launch_bounds__(EngineLayout<N>::THREADS, EngineLayout<N>::MINB)
    k_slice_engine(PassArgs a, EngineArgs e, const __grid_constant__ CUtensorMap tmap)
{
    using L = FftLayout<N>;
    using EL = EngineLayout<N>;
    constexpr int G = L::G, E = L::E, TC = L::TC;
    constexpr int BOX = N < 256 ? N : 256;
    constexpr unsigned TILE_BYTES = (unsigned)(N * TC * sizeof(float2));
    static_assert((size_t)TILE_BYTES <= EL::SCR * sizeof(float2), "the tile lives in the scratch");
    static_assert(L::COL_THREADS == EL::THREADS && EL::ROWS * G == EL::THREADS, "every thread serves both items");
    __shared__ __align__(8) uint64_t bar;
    // the block's loop state, kept in shared memory so that it holds no registers across the
    // transforms: [0] this item's ticket, [1] wait flag, [3] the next ticket, [5] twiddle set in
    // shared memory, [6] the tile barrier's phase (one completion per tile)
    __shared__ int s_item[8];
    // the decoded item (wave, slice, slice index in the launch, item), re-read after the
    // transforms instead of held in registers across them
    __shared__ int s_dec[4];
    auto dec = [&](int i) { return ((volatile int*)s_dec)[i]; };
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float2* smem = reinterpret_cast<float2*>(smem_raw + ((128u - (smem_u32(smem_raw) & 127u)) & 127u));
    float2* tw = smem + EL::SCR;
    float2* etab = tw + N;
    if (ROWOP == ROW_INV_T_FWD) {
        for (int i = threadIdx.x; i < kExpTab; i += blockDim.x) etab[i] = a.exptab[i];
    }
    if (threadIdx.x == 0) {
        mbar_init(&bar, 1);
        s_item[3] = (int)atomicAdd(&e.state->ticket, 1u);
        s_item[5] = -1;
        s_item[6] = 0;
    }
    const long long limit = (a.flags & PF_TEST_WAIT) ? 2000000LL : (e.wait_cycles > 0 ? e.wait_cycles : kWaitCycles);
    const int SUB = e.sub;                              // tiles per item
    const int RI = N / EL::ROWS / SUB, CI = N / TC / SUB;   // row / column items per wave and slice
    // the ticket after this item's: thread 0 takes it once the item's first loads are in flight, so
    // the atomic's latency overlaps them
    auto take_next = [&]() {
        if (threadIdx.x == 0) s_item[3] = (int)atomicAdd(&e.state->ticket, 1u);
    };
    __syncthreads();
    for (;;) {
        if (threadIdx.x == 0) s_item[0] = s_item[3];
        __syncthreads();
        const int t = s_item[0];
        __syncthreads();
        if (t >= e.n_items) break;
        // (slice, phase) of the ticket: phase_start[lo] <= t < phase_start[lo + 1], lo = 2 j + column
        // (a binary search; the table is small and stays in L1)
        int lo = 0;
        {
            int hi = 2 * e.S_max;
            while (hi - lo > 1) {
                const int mid = (lo + hi) >> 1;
                if (e.phase_start[mid] <= t) lo = mid;
                else hi = mid;
            }
        }
        const int j = lo >> 1, s = e.slice0 + j;
        const bool col_item = (lo & 1) != 0;
        const int local = t - e.phase_start[lo];
        const int per = col_item ? CI : RI;
        const int w = local / per, item = local % per;
        if (threadIdx.x == 0) {
            s_dec[0] = w;
            s_dec[1] = s;
            s_dec[2] = j;
            s_dec[3] = item;
        }
        __syncthreads();
        PassArgs as = a;
        as.slice = s;
        if (s >= a.waves[w].n_slices) {
            take_next();   // this wave's slices are done: nothing to do
            continue;
        }
        const int set = s % kTwSets;
        if (!col_item) {
            // ---- row item: SUB blocks of ROWS rows of wave w, slice s
            if (j > 0 && !engine_wait(e.cols_done + w, (unsigned)(j * CI), limit, a.err, &s_item[1])) {
                if (threadIdx.x == 0 && a.err) atomicOr(a.err, 2);
                break;
            }
            // (the barriers at the top of the loop separate the previous item's reads of tw)
            if (set != s_item[5]) {
                for (int i = threadIdx.x; i < N; i += blockDim.x) tw[i] = tw_set<N>(as)[i];
                __syncthreads();
                if (threadIdx.x == 0) s_item[5] = set;
            }
#pragma unroll 1
            for (int k = 0; k < SUB; k++) {
                const int team = threadIdx.x / G, g = threadIdx.x % G;
                float2 v[E];
                {
                    const int r = (dec(3) * SUB + k) * EL::ROWS + team;
                    const float2* src = a.psi + ((size_t)dec(0) * N + r) * N + g;
#pragma unroll
                    for (int q = 0; q < E; q++) v[q] = __ldcg(src + G * q);
                }
                if (k == 0) take_next();
                __syncthreads();
                float2* scr_base = smem + team * L::SCR_STRIDE_ROW;
                auto scr = [scr_base](int k1, int q) { return scr_base + k1 * (G + 1) + q; };
                auto sync = []() { __syncwarp(); };
                conj_all(v);
                team_fft<N, G, -1>(v, g, tw, scr, sync);
                conj_all(v);
                {
                    const int r = (dec(3) * SUB + k) * EL::ROWS + team;
                    const WaveInfo* wi = opaque(a.waves + dec(0));
                    const size_t voff = ((size_t)(dec(1) - a.sV_slice_base) * N + r) * N + g;
                    if (ROWOP == ROW_INV_TT_FWD) {
                        const float2* tr = opaque(a.tt) + (size_t)wi->conf_slot * a.sV_slot_stride + voff;
                        const uint64_t pol = l2_policy_trans(MODE);
#pragma unroll
                        for (int q = 0; q < E; q++) v[q] = cmul(v[q], ld_nc_l2hint(tr + G * q, pol));
                    } else {
                        const float* vr = (wi->sV ? wi->sV : a.sV + (size_t)wi->conf_slot * a.sV_slot_stride) + voff;
#pragma unroll
                        for (int q = 0; q < E; q++) v[q] = cmul(v[q], expi_tab(__ldg(vr + G * q), etab));
                    }
                }
                team_fft<N, G, -1>(v, g, tw, scr, sync);
                const int r = (dec(3) * SUB + k) * EL::ROWS + team;
                float2* dst = opaque(a.psi) + ((size_t)dec(0) * N + r) * N + g;
                const uint64_t pw = l2_policy_wave(MODE);
#pragma unroll
                for (int q = 0; q < E; q++) st_l2hint(dst + G * q, v[q], pw);
            }
            engine_signal(e.rows_done + dec(0));
        } else {
            // ---- column item: SUB tiles of TC columns of wave w, slice s
            // fault injection (PF_TEST_WAIT): the first wave's column items wait for one row item
            // more than the slice has, which no block ever counts
            const unsigned extra = ((a.flags & PF_TEST_WAIT) && w == 0) ? 1u : 0u;
            if (!engine_wait(e.rows_done + w, (unsigned)((j + 1) * RI) + extra, limit, a.err, &s_item[1])) {
                if (threadIdx.x == 0 && a.err) atomicOr(a.err, 2);
                break;
            }
            bool late = false;
#pragma unroll 1
            for (int k = 0; k < SUB; k++) {
                const int col0 = (dec(3) * SUB + k) * TC;
                if (threadIdx.x == 0) {
                    // the tile overwrites shared memory that earlier work used through ordinary
                    // accesses, and reads wave memory that other blocks wrote through ordinary stores
                    asm volatile("fence.proxy.async;" ::: "memory");
                    mbar_expect_tx(&bar, TILE_BYTES);
#pragma unroll
                    for (int q = 0; q < N / BOX; q++)
                        tma_load_2d(smem + q * BOX * TC, &tmap, 2 * col0, dec(0) * N + q * BOX, &bar);
                }
                if (k == 0) {
                    take_next();
                    if (set != s_item[5]) {
                        for (int i = threadIdx.x; i < N; i += blockDim.x) tw[i] = tw_set<N>(as)[i];
                        __syncthreads();
                        if (threadIdx.x == 0) s_item[5] = set;
                    }
                }
                const unsigned phase = (unsigned)s_item[6];
                late = __syncthreads_or(!mbar_wait_bounded(&bar, phase, limit)) != 0;   // block-uniform
                if (late) break;
                const int c = threadIdx.x % TC, g = threadIdx.x / TC;
                float2 v[E];
#pragma unroll
                for (int q = 0; q < E; q++) v[q] = smem[(g + G * q) * TC + c];
                if (threadIdx.x == 0) s_item[6] = (int)(phase ^ 1u);
                __syncthreads();   // every thread holds its values: the tile region becomes the scratch
                float2* scr_base = smem + c * L::SCR_STRIDE_COL;
                auto scr = [scr_base](int k1, int q) { return scr_base + k1 * (G + 1) + q; };
                auto sync = []() { __syncthreads(); };
                const size_t cs = (size_t)G * N;
#pragma unroll 1
                for (int pass = 0; pass < 2; pass++) {
                    team_fft<N, G, -1>(v, g, tw, scr, sync);
                    if (pass == 1) {
                        conj_all(v);
                        break;
                    }
                    const WaveInfo* wi = opaque(a.waves + dec(0));
                    if (dec(1) == wi->n_slices - 1) break;   // the wave's last slice: no propagation
                    const int col = (dec(3) * SUB + k) * TC + c;
                    as.slice = dec(1);
                    const float2* pp = opaque(prop_set(wi->prop ? wi->prop : a.prop, as) + (size_t)g * N + col);
                    const uint64_t pl = l2_policy_evict_last();
#pragma unroll
                    for (int q = 0; q < E; q++) v[q] = cmul(v[q], ld_nc_l2hint(pp + q * cs, pl));
                    conj_all(v);
                }
                const int col = (dec(3) * SUB + k) * TC + c;
                float2* cp = opaque(a.psi + (size_t)dec(0) * N * N + (size_t)g * N + col);
                const uint64_t pw = l2_policy_wave(MODE);
#pragma unroll
                for (int q = 0; q < E; q++) st_l2hint(cp + q * cs, v[q], pw);
                __syncthreads();   // the scratch becomes the next tile
            }
            if (late) {
                if (threadIdx.x == 0 && a.err) atomicOr(a.err, 1);
                break;
            }
            const int wd = dec(0);
            const unsigned done = engine_signal(e.cols_done + wd) + 1u;
            if (threadIdx.x == 0 && dec(1) == a.waves[wd].n_slices - 1 && done == (unsigned)((dec(2) + 1) * CI) &&
                e.done_ns) {
                unsigned long long ns;
                asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(ns));
                e.done_ns[wd] = ns;
            }
        }
    }
}

}  // namespace msb
