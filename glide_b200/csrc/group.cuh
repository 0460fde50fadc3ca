// group.cuh -- grouped launches over several hierarchies.
//
// A group runs the same solver cycle on many independent hierarchies (the
// members of an ensemble, of uneven sizes).  Each member's cycle is recorded
// as its sequence of launches; launches of one kind from different members
// are merged into ONE launch over a table of items, one per
// member: its arguments and its tile grid.  The table is the launch's kernel
// parameters (__grid_constant__, up to 32 KB, read through the constant
// bank).  A block finds its tile's item by a binary search over the table
// from its tile index alone, so the compiler sees the item as uniform over
// the block and reads its arguments as uniform values; a tile whose member
// no longer runs exits at the cost of that search.  By default there is one
// block per tile (k_group); k_group_waves instead runs a fixed number of
// waves of resident blocks that stride over the tiles.  Stencil tiles are staged by
// TMA from the member's own tensor maps, kept in a device array per grouped
// launch (the parameter space holds a pointer to it).
//
// The convergence test of every member runs on the device (k_group_control)
// and clears the member's run flag, so its state stays that of its last
// cycle -- the state a solo solve of that member stops at.
#pragma once

#include <type_traits>

#include "glide_b200.h"
#include "adjoint_kernels.cuh"
#include "forward_kernels.cuh"
#include "tangent_kernels.cuh"
#include "transfer_kernels.cuh"

namespace glide {

// Launch kinds a hierarchy records for grouped execution.
enum GroupOpKind {
    G_SNAPSHOT, G_RESTRICT, G_RESTRICT_BATCH, G_CORRECT_BATCH, G_GROUNDED, G_COPY, G_SET_RHS, G_SWEEP,
    G_RESIDUAL, G_NORMS, G_VJP, G_BLOCK_FACTOR, G_BLOCK_SWEEP, G_GRADIENTS, G_FILL, G_JVP, G_TANGENT_RHS,
    G_NEWTON_UPDATE, G_KINDS
};

template <class R>
struct JvpOpArgs {
    VjpArgs<R> a;
    int mode;
};

struct NormsArgs {
    const double* partial;
    int nblocks;
    double* out;
};

template <class R>
struct RestrictArgs {
    Arr<R> f, c, copy;
    int kind, nyc, nxc;
};

// One item of a grouped launch: the member's grid of gx x gy x gz tiles, as
// its own launch would have it, starting at tile `first` of the launch.
struct GroupItem {
    int first, gx, gy, member;
};

constexpr int kGroupParamBytes = 32000;  // below the 32764-byte kernel parameter limit
constexpr int kGroupMaxItems = 64;        // items of one launch (six steps of the item search at most)

template <class A>
constexpr int group_capacity() {
    return (kGroupParamBytes - 64) / int(sizeof(A) + sizeof(GroupItem)) < kGroupMaxItems
               ? (kGroupParamBytes - 64) / int(sizeof(A) + sizeof(GroupItem))
               : kGroupMaxItems;
}

template <class A, int N>
struct GroupParams {
    const int* flags;            // per-member run flags
    const unsigned char* maps;   // the items' staging maps (BoxMaps), maps_stride apart, or null
    unsigned maps_stride;
    int n;                       // items
    int when;                    // flag bits a member must have for its items to run (0: every member)
    GroupItem item[N];
    A args[N];
};

// The staging maps of one item, in global memory, written by a host copy:
// the acquire fence, at system scope since the writer is the host, orders
// the TMA unit's reads of them after that copy -- an address freed and
// allocated again may still be cached with the maps it held before (thread
// 0 issues the copies, so thread 0 fences).
template <int N>
__device__ __forceinline__ const BoxMaps<N>& item_maps(const unsigned char* mp) {
    const BoxMaps<N>& m = *reinterpret_cast<const BoxMaps<N>*>(mp);
    if (threadIdx.x == 0 && m.use) {
#pragma unroll
        for (int q = 0; q < N; ++q)
            asm volatile("fence.proxy.tensormap::generic.acquire.sys [%0], 128;" ::"l"(&m.m[q]) : "memory");
    }
    return m;
}

// Pointwise kernels: 256 threads, x over columns, y over rows, z over jobs.
template <class R>
struct GSnapshot {
    static constexpr int kMinBlocks = 4;
    using Args = SnapshotArgs<R>;
    static constexpr int kThreads = 256;
    static __device__ __forceinline__ void run(const Args& a, const unsigned char*, GroupBlock b) {
        snapshot_at(a, b.by, b.bx * kThreads + threadIdx.x);
    }
};
template <class R>
struct GRestrict {
    static constexpr int kMinBlocks = 4;
    using Args = RestrictArgs<R>;
    static constexpr int kThreads = 256;
    static __device__ __forceinline__ void run(const Args& a, const unsigned char*, GroupBlock b) {
        restrict_at(a.f, a.c, a.copy, a.kind, a.nyc, a.nxc, b.by, b.bx * kThreads + threadIdx.x);
    }
};
template <class R>
struct GRestrictBatch {
    static constexpr int kMinBlocks = 4;
    using Args = RestrictJobs<R>;
    static constexpr int kThreads = 256;
    static __device__ __forceinline__ void run(const Args& a, const unsigned char*, GroupBlock b) {
        restrict_at(a.f[b.bz], a.c[b.bz], a.copy[b.bz], a.kind[b.bz], a.nyc, a.nxc, b.by,
                    b.bx * kThreads + threadIdx.x);
    }
};
template <class R>
struct GCorrectBatch {
    static constexpr int kMinBlocks = 4;
    using Args = CorrectJobs<R>;
    static constexpr int kThreads = 256;
    static __device__ __forceinline__ void run(const Args& a, const unsigned char*, GroupBlock b) {
        correct_at(a.j[b.bz], b.by, b.bx * kThreads + threadIdx.x);
    }
};
template <class R>
struct GGrounded {
    static constexpr int kMinBlocks = 4;
    using Args = GroundedArgs<R>;
    static constexpr int kThreads = 256;
    static __device__ __forceinline__ void run(const Args& a, const unsigned char*, GroupBlock b) {
        grounded_at(a, b.by, b.bx * kThreads + threadIdx.x);
    }
};
template <class R>
struct GCopy {
    static constexpr int kMinBlocks = 4;
    using Args = CopyArgs<R>;
    static constexpr int kThreads = 256;
    static __device__ __forceinline__ void run(const Args& a, const unsigned char*, GroupBlock b) {
        copy_at(a, b.by, b.bx * kThreads + threadIdx.x);
    }
};
template <class R>
struct GSetRhs {
    static constexpr int kMinBlocks = 4;
    using Args = SetRhsArgs<R>;
    static constexpr int kThreads = 256;
    static __device__ __forceinline__ void run(const Args& a, const unsigned char*, GroupBlock b) {
        set_rhs_at(a, b.by, b.bx * kThreads + threadIdx.x);
    }
};
template <class R>
struct GGradients {
    static constexpr int kMinBlocks = 4;
    using Args = GradArgs<R>;
    static constexpr int kThreads = 256;
    static __device__ __forceinline__ void run(const Args& a, const unsigned char*, GroupBlock b) {
        const int J = b.bx * kThreads + threadIdx.x;
        if (J < a.nx) gradients_at(a, b.by, J);
    }
};
template <class R>
struct GFill {
    static constexpr int kMinBlocks = 4;
    using Args = FillArgs<R>;
    static constexpr int kThreads = 256;
    static __device__ __forceinline__ void run(const Args& a, const unsigned char*, GroupBlock b) {
        fill_at(a, b.by, b.bx * kThreads + threadIdx.x);
    }
};
template <class R>
struct GTangentRhs {
    static constexpr int kMinBlocks = 4;
    using Args = TangentRhsArgs<R, R>;
    static constexpr int kThreads = 256;
    static __device__ __forceinline__ void run(const Args& a, const unsigned char*, GroupBlock b) {
        tangent_rhs_at(a, b.by, b.bx * kThreads + threadIdx.x);
    }
};
template <class R>
struct GNewtonUpdate {
    static constexpr int kMinBlocks = 4;
    using Args = NewtonUpdateArgs<R, R>;
    static constexpr int kThreads = 256;
    static __device__ __forceinline__ void run(const Args& a, const unsigned char*, GroupBlock b) {
        newton_update_at(a, b.by, b.bx * kThreads + threadIdx.x);
    }
};
struct GNorms {
    static constexpr int kMinBlocks = 1;
    using Args = NormsArgs;
    static constexpr int kThreads = kNormThreads;
    static __device__ __forceinline__ void run(const Args& a, const unsigned char*, GroupBlock) {
        finish_norms_block(a.partial, a.nblocks, a.out);
    }
};

// Stencil kernels: the tile bodies of the per-hierarchy kernels, staged from
// the item's maps (kMaps of them).  A block re-initialises the staging
// mbarrier for every tile it runs; the tiles are separated by a block-wide
// barrier, so no thread still waits on the previous phase.
template <class Op, class = void>
struct OpMaps {
    static constexpr int n = 0;
};
template <class Op>
struct OpMaps<Op, std::void_t<decltype(Op::kMaps)>> {
    static constexpr int n = Op::kMaps;
};

// Register budgets: the per-hierarchy kernels' resident blocks per SM.
template <class R, bool PHI_LIVE, int MINB>
struct GSweep {
    static constexpr int kMinBlocks = MINB;
    using Args = SweepArgs<R>;
    static constexpr int kThreads = kSweepThreads;
    static __device__ __forceinline__ void run(const Args& a, const unsigned char*, GroupBlock b) {
        vanka_sweep_tile<R, PHI_LIVE>(a, a.gmode, b);
    }
};
template <class R>
struct GResidual {
    static constexpr int kMaps = 7;
    static constexpr int kMinBlocks = sizeof(R) == 8 ? 4 : 5;
    using Args = ResidualArgs<R>;
    static constexpr int kThreads = 256;
    static __device__ __forceinline__ void run(const Args& a, const unsigned char* mp, GroupBlock b) {
        residual_tile<R>(a, item_maps<7>(mp), b);
    }
};
template <class R>
struct GVjp {
    static constexpr int kMaps = 9;
    static constexpr int kMinBlocks = sizeof(R) == 8 ? 2 : 3;
    using Args = VjpArgs<R>;
    static constexpr int kThreads = kTileA * kTileA;
    static __device__ __forceinline__ void run(const Args& a, const unsigned char* mp, GroupBlock b) {
        vjp_tile<R>(a, item_maps<9>(mp), b);
    }
};
template <class R>
struct GJvp {
    static constexpr int kMaps = JvpTile<R>::NB;
    static constexpr int kMinBlocks = sizeof(R) == 8 ? 3 : 6;
    using Args = JvpOpArgs<R>;
    static constexpr int kThreads = kTileA * kTileA;
    static __device__ __forceinline__ void run(const Args& a, const unsigned char* mp, GroupBlock b) {
        jvp_tile<R>(a.a, a.mode, item_maps<JvpTile<R>::NB>(mp), b);
    }
};
template <class R, bool TR>
struct GBlockFactor {
    static constexpr int kMaps = 7;
    static constexpr int kMinBlocks = sizeof(R) == 8 ? 2 : 4;
    using Args = BlockArgs<R>;
    static constexpr int kThreads = kTile * kTile;
    static __device__ __forceinline__ void run(const Args& a, const unsigned char* mp, GroupBlock b) {
        block_factor_tile<R, TR>(a, item_maps<7>(mp), b);
    }
};
template <class R, bool TR>
struct GBlockSweep {
    static constexpr int kMinBlocks = sizeof(R) == 8 ? 4 : 5;
    using Args = BlockArgs<R>;
    static constexpr int kThreads = kSweepThreads;
    static __device__ __forceinline__ void run(const Args& a, const unsigned char*, GroupBlock b) {
        block_sweep_tile<R, TR>(a, b);
    }
};

// The item holding tile t: the last item whose range starts at or before t.
template <class A, int N>
__device__ __forceinline__ int group_item_of(const GroupParams<A, N>& P, int t) {
    int lo = 0, hi = P.n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (P.item[mid].first <= t) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// One block per tile of all items.
template <class Op, int N>
__global__ void __launch_bounds__(Op::kThreads, Op::kMinBlocks)
    k_group(const __grid_constant__ GroupParams<typename Op::Args, N> P) {
    const int t = int(blockIdx.x);
    const int k = group_item_of(P, t);
    const GroupItem& it = P.item[k];
    if (P.when && (P.flags[it.member] & P.when) == 0) return;  // uniform over the block
    const unsigned gx = unsigned(it.gx), local = unsigned(t - it.first), per = gx * unsigned(it.gy);
    const unsigned rest = local % per;
    Op::run(P.args[k], P.maps + size_t(k) * P.maps_stride, GroupBlock{rest % gx, rest / gx, local / per, gx});
}

// `total` tiles of all items, strided over by a fixed grid; the loop and the
// item search depend only on blockIdx and the parameters.
template <class Op, int N>
__global__ void __launch_bounds__(Op::kThreads, Op::kMinBlocks)
    k_group_waves(const __grid_constant__ GroupParams<typename Op::Args, N> P, int total) {
    for (int t = blockIdx.x; t < total; t += gridDim.x) {
        const int k = group_item_of(P, t);
        const GroupItem& it = P.item[k];
        if (P.when && (P.flags[it.member] & P.when) == 0) continue;  // uniform over the block
        const unsigned gx = unsigned(it.gx), local = unsigned(t - it.first), per = gx * unsigned(it.gy);
        const unsigned rest = local % per;
        Op::run(P.args[k], P.maps + size_t(k) * P.maps_stride, GroupBlock{rest % gx, rest / gx, local / per, gx});
        __syncthreads();  // the next tile restages the block's shared memory
    }
}

// ------------------------------------------------------------ convergence
// Per-member solve state on the device, and the per-hierarchy solve loop's
// decisions taken there (Solver::solve_loop): another cycle while
// rel > rtol, |r| > atol and cycles < max; on a forward solve with the Newton
// method, a Newton step once rel <= newton_switch and rel <= gate, preceded
// by the Newton prologue when the previous cycle was not one, its state saved
// first and restored if the residual grew (gate then drops tenfold), and
// Newton switched off after two steps that cut the residual by less than the
// stall ratio.  A cycle's launches are predicated on the member's flag bits.
constexpr int kGroupHistory = GLIDE_MAX_HISTORY;
enum GroupFlag {
    kGroupRun = 1,     // the member runs this cycle
    kGroupFas = 2,     // ... a FASCD cycle (or a linear cycle)
    kGroupNewton = 4,  // ... a Newton step (saved state, tangent solve, update)
    kGroupPro = 8,     // ... preceded by the Newton prologue
    kGroupUndo = 16,   // the Newton step is undone
};
enum GroupStatus { GS_RUNNING = 0, GS_DONE = 1, GS_NONFINITE = 2, GS_STAGING = 3 };
enum GroupPhase { GC_INIT = 0, GC_MID = 1, GC_POST = 2, GC_END = 3 };

struct GroupMember {
    const double* norms;  // the member's norm vector |r_u|, |r_v|, |r_H|, |r|
    const int* err;       // the member's error word (kStage* bits of a staging block)
    int err_word;         // its value when the member stopped on it
    double rtol, atol;
    double newton_switch, stall_ratio;
    int max_cycles;
    int newton;           // forward solve with the Newton method
    int cycles, status;
    int in_newton, newton_off, stall, rejects;
    int fas_cycles, prologues;  // cycles that were FASCD (or linear) cycles; Newton prologues run
    double r0, last, rel, prev, gate;
    double last_norms[3];
    double history[kGroupHistory];
};

constexpr int kGroupControlThreads = 1024;

// The next cycle of a running member: a Newton step or a FASCD cycle, with
// the Newton prologue when the previous cycle was not a Newton step.
__device__ __forceinline__ int group_decide(GroupMember& g) {
    const bool newton_phase = g.newton && g.rel <= g.newton_switch;
    const bool step = newton_phase && !g.newton_off && g.rel <= g.gate;
    if (!step) g.in_newton = 0;
    return kGroupRun | (step ? kGroupNewton : kGroupFas) | (step && !g.in_newton ? kGroupPro : 0);
}

// One phase of the decisions for every member (one thread each); GC_INIT and
// GC_END also decide every running member's next cycle.  Members that stopped
// are left alone.  After GC_INIT and GC_END, out[0] is the number of members
// still running and out[1] the union of their next cycle's section bits.
__global__ void __launch_bounds__(kGroupControlThreads)
    k_group_control(GroupMember* m, int* flags, int n, int phase, int* out) {
    __shared__ int count, sections;
    if (threadIdx.x == 0) count = sections = 0;
    __syncthreads();
    for (int k = threadIdx.x; k < n; k += blockDim.x) {
        GroupMember& g = m[k];
        int f = flags[k];
        if (phase == GC_INIT) {
            const double ab = g.norms[3];
            g.r0 = g.last = g.prev = ab;
            g.rel = 1.0;
            g.gate = g.newton_switch;
            g.cycles = g.fas_cycles = g.prologues = 0;
            g.in_newton = g.newton_off = g.stall = g.rejects = 0;
            g.history[0] = ab;
            for (int q = 0; q < 3; ++q) g.last_norms[q] = g.norms[q];
            if (const int e = *(volatile const int*)g.err) {  // the norms are not this residual's
                g.status = GS_STAGING;
                g.err_word = e;
                f = 0;
            } else if (!isfinite(ab)) {
                g.status = GS_NONFINITE;
                f = 0;
            } else {
                const bool run = g.rel > g.rtol && ab > g.atol && g.max_cycles > 0;
                g.status = run ? GS_RUNNING : GS_DONE;
                f = run ? group_decide(g) : 0;
            }
        } else if (!(f & kGroupRun)) {
            continue;
        } else if (phase == GC_MID) {
            if (f & kGroupPro) {
                g.prev = g.norms[3];
                g.in_newton = 1;
                g.prologues += 1;
            }
        } else if (phase == GC_POST) {
            if ((f & kGroupNewton) && !(g.norms[3] <= g.prev)) f |= kGroupUndo;
        } else {  // GC_END
            if (const int e = *(volatile const int*)g.err) {
                g.status = GS_STAGING;
                g.err_word = e;
                flags[k] = 0;
                continue;
            }
            double ab = g.norms[3];
            for (int q = 0; q < 3; ++q) g.last_norms[q] = g.norms[q];
            if (f & kGroupUndo) {
                ab = g.prev;
                g.gate = 0.1 * (g.prev / g.r0);
                g.in_newton = 0;
                g.stall = 0;
                g.rejects += 1;
            }
            if (!isfinite(ab)) {
                g.status = GS_NONFINITE;
                g.last = ab;
                flags[k] = 0;
                continue;
            }
            g.rel = ab / g.r0;
            if ((f & kGroupNewton) && g.in_newton) {
                g.stall = ab > g.stall_ratio * g.prev ? g.stall + 1 : 0;
                if (g.stall >= 2) g.newton_off = 1;
            }
            g.prev = ab;
            g.last = ab;
            g.cycles += 1;
            if (!(f & kGroupNewton)) g.fas_cycles += 1;
            if (g.cycles < kGroupHistory) g.history[g.cycles] = ab;
            const bool run = g.rel > g.rtol && ab > g.atol && g.cycles < g.max_cycles;
            g.status = run ? GS_RUNNING : GS_DONE;
            f = run ? group_decide(g) : 0;
        }
        flags[k] = f;
        if (f & kGroupRun) {
            atomicAdd(&count, 1);
            atomicOr(&sections, f);
        }
    }
    __syncthreads();
    if (threadIdx.x == 0 && (phase == GC_INIT || phase == GC_END)) {
        out[0] = count;
        out[1] = sections;
    }
}

}  // namespace glide
