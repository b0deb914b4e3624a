// Persistent multi-shot 2D kernel: the batches of several shots advance together in one launch
// driven by a (shot, tile, stage) work queue.
//
// The work of a launch is a list of items in a fixed global order: for each step j of the
// batch, for each phase (RK stages 0-3, then the verdict), for each shot still stepping at j
// (shots sorted by batch length, longest first), the shot's stage tiles (or its one verdict
// item).  A resident CTA takes the next item with an atomic ticket, waits until the items it
// depends on have finished (per-tile counters for the 3x3 tiles of the previous stage; per-shot
// counters for a verdict and for stage 0 after it), runs it -- a stage tile is
// exactly the tile the per-shot stage kernel runs, a verdict is the per-shot verdict kernel's
// reduction, acceptance rule, receiver record and clock advance -- and counts it done.  Items are
// taken in order and an item only waits on items earlier in the order, all of which were taken
// by CTAs that are running, so the queue always drains; every wait is bounded all the same, and
// one that runs out stops the launch with an error word the host reports.  A tile starts its next
// stage as soon as its neighbours finished theirs, so stages overlap within a shot, and the tiles
// of the other shots keep the SMs busy while one shot waits at its verdict.
#pragma once
#include "stage2d.cuh"

namespace swl::k2 {

// One shot of a queued batch (device copy, written by the host before the launch).
template <class Real> struct QueueShot {
    StageArgs<Real> stage[2][4]; // [set holding the step's start state U][RK stage]
    Partial *partials;           // per-tile diagnostics of stage 3 (the verdict reduces them)
    const long long *receivers;
    double *traces;
    Clock *clock;
    const Real *sets[2]; // state sets 0 and 1: a step that starts from set r leaves its new state in set 1 - r
    long long count;     // stride between fields
    int nrec, tiles, tilesX, u0, steps, first;
};

// Launch-wide queue state and order tables.
struct QueueHeader {
    unsigned long long head;      // next ticket
    unsigned long long total;     // items in the launch
    int abort;                    // 0 running; 1 a copy wait ran out; 2 a dependency wait ran out
    int nshots, maxSteps, pad;
    int *done;                    // [nshots] items finished per shot
    int *progress;                // [tilePrefix[nshots]] stage items finished per tile (tilePrefix[s] + tile)
    const long long *stepStart;   // [maxSteps + 1] first item of step j
    const int *active;            // [maxSteps] shots stepping at step j (a prefix of the shot order)
    const long long *tilePrefix;  // [nshots + 1] stage tiles of the shots before shot s
};

// The MacCormack direction of axis x (0) or z (1) at (step, stage): the x and z columns of the
// 8-step table of include/SeisCommon/FiniteDifference.hpp:9-13 (backward x in rows 1, 2, 5, 6;
// backward z in rows 2, 3, 6, 7), flipped at each RK stage.
__device__ __forceinline__ int queueDirection(int step, int stage, int axis) {
    return int(((axis ? 0xCCu : 0x66u) >> (step & 7)) + unsigned(stage)) & 1;
}

__device__ __forceinline__ int ldAcquire(const int *p) {
    int v;
    asm volatile("ld.acquire.gpu.global.s32 %0, [%1];\n" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void redRelease(int *p, int v) {
    asm volatile("red.release.gpu.global.add.s32 [%0], %1;\n" ::"l"(p), "r"(v) : "memory");
}
// Generic-proxy writes and reads ordered with the tensor copies (async proxy) of the same data.
__device__ __forceinline__ void fenceProxyAsync() { asm volatile("fence.proxy.async.global;\n" ::: "memory"); }
// A tensor map the host copied into global memory, acquired for the tensor copies that use it.
__device__ __forceinline__ void fenceTensorMap(const CUtensorMap *map) {
    asm volatile("fence.proxy.tensormap::generic.acquire.sys [%0], 128;\n" ::"l"(map) : "memory");
}
__device__ __forceinline__ unsigned long long globalTimer() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %globaltimer;\n" : "=l"(t));
    return t;
}

// The verdict of one step of one shot (verdict2d with its 1024-thread reduction tree, run by the
// 256 threads of a CTA over `sh`, 1024 partials of shared memory, so the sums are the same).
template <class Real>
__device__ __forceinline__ void queueVerdict(const QueueShot<Real> &q, const Real *w, Partial *sh) {
    constexpr int V = 1024, T = STREAM_THREADS;
    __shared__ int accept;
    const int t = threadIdx.x + SW * threadIdx.y;
    Clock *clk = q.clock;
    if (clk->faulted) return; // uniform: every thread reads the same word after the dependency wait
    for (int v = t; v < V; v += T) {
        Partial s{0, 0, 0, 0, 0};
        for (int b = v; b < q.tiles; b += V) {
            const Partial y = q.partials[b];
            s.energy += y.energy;
            s.velocity = fmax(s.velocity, y.velocity);
            s.traction = fmax(s.traction, y.traction);
            s.bad |= y.bad;
        }
        sh[v] = s;
    }
    __syncthreads();
    for (int stride = V / 2; stride > 0; stride >>= 1) {
        for (int v = t; v < stride; v += T) {
            Partial &x = sh[v];
            const Partial y = sh[v + stride];
            x.energy += y.energy;
            x.velocity = fmax(x.velocity, y.velocity);
            x.traction = fmax(x.traction, y.traction);
            x.bad |= y.bad;
        }
        __syncthreads();
    }
    if (t == 0) {
        const Partial tot = sh[0];
        const bool finite = !tot.bad && isfinite(tot.energy);
        const bool growth =
            (clk->step + 1) * clk->dt > clk->growth_after && clk->peak_energy > 0 && tot.energy > clk->peak_energy * 10000;
        const int ok = finite && !growth;
        clk->finite = finite;
        if (ok) {
            clk->energy = tot.energy;
            clk->max_velocity = tot.velocity;
            clk->traction = tot.traction;
            clk->peak_energy = fmax(clk->peak_energy, tot.energy);
        }
        accept = ok;
    }
    __syncthreads();
    if (!accept) {
        if (t == 0) {
            clk->faulted = 1;
            clk->fault_step = clk->step;
        }
        return;
    }
    const int row = clk->step - clk->first;
    if (row < clk->trace_steps)
        for (int r = t; r < q.nrec; r += T) {
            const long long qq = q.receivers[r];
            q.traces[((long long)row * q.nrec + r) * 2] = double(w[qq]);
            q.traces[((long long)row * q.nrec + r) * 2 + 1] = double(w[q.count + qq]);
        }
    __syncthreads();
    if (t == 0) {
        clk->step += 1;
        clk->accepted += 1;
    }
}

template <class Real, int MECH, int DX, int DZ>
__device__ __forceinline__ bool queueStage(const StageArgs<Real> &p, int stage, uint64_t *bar, Real *ring, Real *pw, int bx, int by,
                                           int slot, bool reinit) {
    switch (stage) {
    case 0: return streamTile<Real, DX, DZ, MECH, 0>(p, bar, ring, pw, bx, by, slot, reinit);
    case 1: return streamTile<Real, DX, DZ, MECH, 1>(p, bar, ring, pw, bx, by, slot, reinit);
    case 2: return streamTile<Real, DX, DZ, MECH, 2>(p, bar, ring, pw, bx, by, slot, reinit);
    default: return streamTile<Real, DX, DZ, MECH, 3>(p, bar, ring, pw, bx, by, slot, reinit);
    }
}

// Bound of one dependency wait: far longer than any phase of any shot takes.
constexpr unsigned long long kQueueWaitNs = 4000000000ull;
// Shots per launch.
constexpr int kQueueMaxShots = 256;

// Resident CTAs per SM: the stage kernels' count.  (Two CTAs of the GSLS forms, which would keep
// their values in registers, measured slower than three with a few hundred bytes of spills.)
template <class Real, int MECH> constexpr int queueBlocks() { return streamBlocks<Real>(); }

template <class Real, int MECH>
__global__ void __launch_bounds__(STREAM_THREADS, (queueBlocks<Real, MECH>())) queue2d(QueueHeader *hdr, const QueueShot<Real> *shots) {
    extern __shared__ __align__(16) unsigned char smemRaw[];
    unsigned char *base = smemRaw + ((128 - (smemAddr(smemRaw) & 127)) & 127);
    uint64_t *bar = reinterpret_cast<uint64_t *>(base);
    Real *ring = reinterpret_cast<Real *>(base + 128);
    Real *pw = ring + CHUNKS * CH;
    __shared__ unsigned long long item;
    __shared__ int go, ready;
    __shared__ unsigned fenced[kQueueMaxShots * 8 / 32]; // tensor maps this CTA acquired: (shot, set, stage)
    const int tid = threadIdx.x + SW * threadIdx.y;
    for (int w = tid; w < kQueueMaxShots * 8 / 32; w += STREAM_THREADS) fenced[w] = 0;
    bool used = false; // the mbarriers hold an earlier tile's (completed) phases
    for (;;) {
        if (tid == 0) {
            item = atomicAdd(&hdr->head, 1ull);
            go = item < hdr->total && !*(volatile int *)&hdr->abort;
        }
        __syncthreads();
        if (!go) break;
        const unsigned long long it = item;
        // decode: step j (binary search of the step starts), phase, shot, tile
        int lo = 0, hi = hdr->maxSteps; // stepStart[lo] <= it < stepStart[hi]
        while (hi - lo > 1) {
            const int mid = (lo + hi) >> 1;
            if ((unsigned long long)__ldg(hdr->stepStart + mid) <= it) lo = mid;
            else hi = mid;
        }
        const int j = lo, act = __ldg(hdr->active + j);
        const long long o = (long long)(it - (unsigned long long)__ldg(hdr->stepStart + j));
        const long long perStage = __ldg(hdr->tilePrefix + act);
        int phase, s;
        long long tile = 0;
        if (o < 4 * perStage) {
            phase = int(o / perStage);
            const long long r = o - phase * perStage;
            int a = 0, b = act; // tilePrefix[a] <= r < tilePrefix[b]
            while (b - a > 1) {
                const int mid = (a + b) >> 1;
                if (__ldg(hdr->tilePrefix + mid) <= r) a = mid;
                else b = mid;
            }
            s = a;
            tile = r - __ldg(hdr->tilePrefix + a);
        } else {
            phase = 4;
            s = int(o - 4 * perStage);
        }
        const QueueShot<Real> &q = shots[s];
        const int bx = int(tile % q.tilesX), by = int(tile / q.tilesX);
        int *const prog = hdr->progress + __ldg(hdr->tilePrefix + s);
        // Dependencies.  Stages 1-3 of a tile read the previous stage's output of the 3x3 tiles
        // around it (the stencil halo is 4 columns and 3 rows, less than a tile) and overwrite
        // what that stage read there, so they wait for those nine tiles only.  A verdict waits for
        // every stage-3 tile of its step; stage 0 of a step waits for the previous verdict (the
        // new state, the clock and a possible rejection), which covers everything before it.
        if (tid < 32) {
            int state = 1; // 1 ready, 0 stop
            if (phase >= 1 && phase <= 3) {
                const int need = 4 * j + phase;
                const int tilesY = q.tiles / q.tilesX;
                const int nx = bx + tid % 3 - 1, ny = by + tid / 3 - 1;
                const bool mine = tid < 9 && nx >= 0 && nx < q.tilesX && ny >= 0 && ny < tilesY;
                const int *flag = prog + (mine ? ny * q.tilesX + nx : 0);
                if (!__all_sync(0xffffffffu, !mine || ldAcquire(flag) >= need)) {
                    const unsigned long long t0 = globalTimer();
                    unsigned ns = 32;
                    for (;;) {
                        __nanosleep(ns);
                        ns = ns < 1024 ? 2 * ns : ns;
                        if (__all_sync(0xffffffffu, !mine || ldAcquire(flag) >= need)) break;
                        int stop = 0;
                        if (tid == 0) {
                            if (*(volatile int *)&hdr->abort) stop = 1;
                            else if (globalTimer() - t0 > kQueueWaitNs) atomicCAS(&hdr->abort, 0, 2), stop = 1;
                        }
                        if (__shfl_sync(0xffffffffu, stop, 0)) {
                            state = 0;
                            break;
                        }
                    }
                }
            } else if (tid == 0) {
                const int need = j * (4 * q.tiles + 1) + phase * q.tiles;
                if (ldAcquire(hdr->done + s) < need) {
                    const unsigned long long t0 = globalTimer();
                    unsigned ns = 32;
                    for (;;) {
                        __nanosleep(ns);
                        ns = ns < 1024 ? 2 * ns : ns;
                        if (ldAcquire(hdr->done + s) >= need) break;
                        if (*(volatile int *)&hdr->abort) {
                            state = 0;
                            break;
                        }
                        if (globalTimer() - t0 > kQueueWaitNs) {
                            atomicCAS(&hdr->abort, 0, 2);
                            state = 0;
                            break;
                        }
                    }
                }
            }
            if (tid == 0) ready = state;
        }
        if (tid == 0) {
            asm volatile("fence.acq_rel.gpu;\n" ::: "memory"); // what the waiting lanes acquired, for the whole CTA
            fenceProxyAsync(); // the tensor copies below read what other CTAs wrote
            if (phase < 4) { // the maps of this (shot, set, stage), once per CTA and launch
                const int set = (j & 1) ? 1 - q.u0 : q.u0, bit = (s * 2 + set) * 4 + phase;
                if (!(fenced[bit >> 5] & (1u << (bit & 31)))) {
                    const StageArgs<Real> &p = q.stage[set][phase];
                    fenceTensorMap(&p.ringMap), fenceTensorMap(&p.uMap), fenceTensorMap(&p.aMap);
                    fenceTensorMap(&p.modelMap), fenceTensorMap(&p.compMap);
                    fenced[bit >> 5] |= 1u << (bit & 31);
                }
            }
        }
        __syncthreads();
        if (!ready) break;
        bool ok = true;
        const int step = q.first + j;
        const int r = (j & 1) ? 1 - q.u0 : q.u0; // set holding step j's start state
        if (phase == 4) {
            queueVerdict<Real>(q, q.sets[1 - r], reinterpret_cast<Partial *>(ring));
        } else if (!q.clock->faulted) {
            const StageArgs<Real> &p = q.stage[r][phase];
            const int dx = queueDirection(step, phase, 0), dz = queueDirection(step, phase, 1);
            if (dx == 0 && dz == 0) ok = queueStage<Real, MECH, 0, 0>(p, phase, bar, ring, pw, bx, by, int(tile), used);
            else if (dx == 0) ok = queueStage<Real, MECH, 0, 1>(p, phase, bar, ring, pw, bx, by, int(tile), used);
            else if (dz == 0) ok = queueStage<Real, MECH, 1, 0>(p, phase, bar, ring, pw, bx, by, int(tile), used);
            else ok = queueStage<Real, MECH, 1, 1>(p, phase, bar, ring, pw, bx, by, int(tile), used);
            used = true;
        }
        fenceProxyAsync(); // this item's writes, before they are published to later copies
        __syncthreads();
        if (tid == 0) { // publish: the barrier orders the CTA's writes before these releases
            if (!ok) atomicCAS(&hdr->abort, 0, 1);
            if (phase < 4) redRelease(prog + tile, 1);
            redRelease(hdr->done + s, 1);
        }
    }
}

} // namespace swl::k2
