// runtime.cu -- level hierarchy, FASCD / FASAdjoint drivers and the C ABI.
//
// One handle owns the whole multigrid hierarchy in a single device arena:
// every level's state, parameters, operator arrays and V-cycle scratch, each
// 2-D array with its row pitch rounded up to 32 elements and its start aligned
// to 256 bytes (coalesced rows; TMA-legal strides).  The V-cycle schedule runs
// here, in C++, issuing fused kernels on the caller's stream; with graphs on,
// one V-cycle plus its convergence-check residual is captured once and
// replayed, so a solve costs one host synchronisation per V-cycle.
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <cmath>
#include <functional>
#include <mutex>
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "glide_b200.h"
#include "forward_kernels.cuh"
#include "adjoint_kernels.cuh"
#include "tangent_kernels.cuh"
#include "transfer_kernels.cuh"
#include "group.cuh"

namespace glide {

// ------------------------------------------------------------------ errors
static thread_local std::string g_err;

// Stream captures of CUDA graphs and the device allocations made while
// solving take this lock: handles driven from several host threads then never
// allocate while another thread's capture is open, nor open two at once.
static std::mutex g_capture_mu;

struct Fail {
    int code;
};

[[noreturn]] static void fail(int code, const std::string& msg) {
    g_err = msg;
    throw Fail{code};
}

#define GCU(call)                                                                       \
    do {                                                                                \
        cudaError_t e_ = (call);                                                        \
        if (e_ != cudaSuccess)                                                          \
            fail(GLIDE_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_));   \
    } while (0)

static void check_launch(const char* what) {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) fail(GLIDE_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

__global__ void __launch_bounds__(kNormThreads) k_finish_norms(const double* partial, int nblocks, double* out) {
    finish_norms_block(partial, nblocks, out);
}

// ------------------------------------------------------------------ fields
enum InternalField {
    F_U_ALT = GLIDE_N_PUBLIC_FIELDS, F_V_ALT, F_H_ALT,
    F_W_U, F_W_V, F_W_H, F_CHI,
    F_WL_U, F_WL_V, F_WL_H,
    // tangent (Newton correction) system: correction, right-hand side,
    // residual and the coarse-level snapshot of the correction
    F_E_U, F_E_V, F_E_H, F_TF_U, F_TF_V, F_TF_H, F_TR_U, F_TR_V, F_TR_H, F_TW_U, F_TW_V, F_TW_H,
    // state before a Newton step, restored when the step is rejected
    F_BK_U, F_BK_V, F_BK_H, F_BK_MASK,
    F_COUNT
};

enum Kind { KU = 0, KV = 1, KC = 2 };

static Kind field_kind(int f) {
    switch (f) {
        case GLIDE_U: case GLIDE_F_U: case GLIDE_R_U: case GLIDE_LAMBDA_U: case GLIDE_ADJ_F_U:
        case GLIDE_ADJ_R_U: case GLIDE_VJP_U: case GLIDE_FOP_U: case F_U_ALT: case F_W_U: case F_WL_U:
        case F_E_U: case F_TF_U: case F_TR_U: case F_TW_U: case GLIDE_VAR_U: case GLIDE_JVP_U:
        case F_BK_U:
            return KU;
        case GLIDE_V: case GLIDE_F_V: case GLIDE_R_V: case GLIDE_LAMBDA_V: case GLIDE_ADJ_F_V:
        case GLIDE_ADJ_R_V: case GLIDE_VJP_V: case GLIDE_FOP_V: case F_V_ALT: case F_W_V: case F_WL_V:
        case F_E_V: case F_TF_V: case F_TR_V: case F_TW_V: case GLIDE_VAR_V: case GLIDE_JVP_V:
        case F_BK_V:
            return KV;
        default:
            return KC;
    }
}

static glide_phys default_phys() {
    glide_phys p;
    p.n = 3.0; p.eps_reg = 1e-6; p.flotation_reg_driving = 0.1; p.m = 1.0; p.u_reg = 1.0;
    p.water_drag = 1e-5; p.flotation_reg_sliding = 0.1; p.calving_rate = 0.0;
    p.flotation_reg_calving = 0.1; p.thklim = 0.1;
    return p;
}

static glide_fas_config default_fas() {
    glide_fas_config c;
    c.freeze_coarse_calving = 1; c.freeze_coarse_phi = 1;
    c.coarsest_steps = 200; c.pre_steps = 10; c.post_steps = 20; c.finest_steps = 50;
    c.maximum_vcycles = 10; c.relative_tolerance = 1e-3; c.absolute_tolerance = 5.0;
    return c;
}

static glide_vanka_config default_vanka() {
    glide_vanka_config c;
    c.omega = 0.5; c.newton_steps = 30; c.relaxation = 0.5; c.ssa_damping = 0.01;
    c.mc_damping = 1.0; c.relax_phi = 0.0;
    return c;
}

// Linear multigrid of the Newton correction: light smoothing, no extra
// finest-level sweeps; block smoother with the forward damping and omega 0.8.
static glide_fas_config default_tangent_fas() {
    glide_fas_config c = default_fas();
    c.coarsest_steps = 50; c.pre_steps = 4; c.post_steps = 4; c.finest_steps = 0;
    return c;
}

static glide_vanka_config default_tangent_vanka() {
    glide_vanka_config c = default_vanka();
    c.omega = 0.8;
    return c;
}

static int round_up(int a, int m) { return (a + m - 1) / m * m; }

// the arrays of a StateBoxTile, in its staging order
static constexpr int kStateBoxes[7] = {GLIDE_U, GLIDE_V, GLIDE_H, GLIDE_PHI, GLIDE_BED, GLIDE_BETA, GLIDE_B};

// cuTensorMapEncodeTiled from the driver, looked up once through the runtime
// (the library links only libcudart)
static PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    });
    return fn;
}

struct SolverBase {
    virtual ~SolverBase() {}
    int dtype = GLIDE_F64;
    int n_levels = 0;
    // [0] forward FASCD, [1] FASAdjoint, [2] tangent (Newton correction) multigrid
    glide_fas_config fas[3];
    int quirks = 1;
    int use_graphs = 1;
    unsigned version = 1;
    // Vanka sweep register budget: resident blocks per SM (1 or 2)
    int sweep_blocks_per_sm = 2;
    // forward solve: 0 = FASCD V-cycles only (the reference's method);
    // 1 = FASCD until rel. residual <= newton_switch, then Newton steps whose
    //     correction comes from the tangent linear multigrid
    int forward_method = 0;
    double newton_switch = 1e-2;
    double newton_stall_ratio = 0.7;
};

// A launch recorded instead of issued, for grouped execution: the kind and
// template variant, the grid the per-hierarchy launch would use, the argument
// struct's bytes and the launch's algorithmic bytes.
struct RecOp {
    int op, variant;
    int gx, gy, gz;
    std::vector<unsigned char> args;
    double bytes;
    std::vector<unsigned char> maps;  // the staging maps of a stencil launch (BoxMaps)
};

template <class R>
struct Solver;

template <class R>
struct Level {
    int ny = 0, nx = 0;
    double dx = 0;
    int pu = 0, pv = 0, pc = 0;
    Arr<R> a[F_COUNT];
    glide_phys phys;
    glide_vanka_config vk[3];  // [0] forward, [1] adjoint, [2] tangent
    int blocks_x() const { return (nx + kTile - 1) / kTile; }
    int blocks_y() const { return (ny + kTile - 1) / kTile; }
};

template <class R>
struct Solver : SolverBase {
    std::vector<Level<R>> lv;
    char* arena = nullptr;
    double* partial = nullptr;
    double* norms_dev = nullptr;
    double* norms_host = nullptr;
    int* err_dev = nullptr;  // kStage* bits set by a staging block (its wait gave up, or its maps failed their check)
    // TMA tensor maps of every (level, field), encoded on first use
    // slot per box height (kTmaHeights)
    static constexpr int kTmaHeights[3] = {kBoxH, 22, 24};
    std::vector<CUtensorMap> tmaps[3];
    std::vector<unsigned char> tmap_done[3];
    bool use_tma = true;
    int tma_wait_polls = kTmaWaitPolls;  // 0 under GLIDE_TUNE_TMA_GIVE_UP
    // one captured V-cycle per cycle kind (0 FAS, 1 adjoint, 2 mixed FAS,
    // 3 mixed adjoint, 4 Newton), each valid for the (version, dt, start) it
    // was captured with, so that solves alternating kinds replay, not recapture
    static constexpr int kKinds = 5;
    struct CachedGraph {
        cudaGraphExec_t exec = nullptr;
        unsigned version = 0;
        double dt = 0;
        int start = -1;
        long long launches = 0;  // kernels inside the graph
        double bytes = 0;        // their algorithmic bytes
    };
    CachedGraph graphs[kKinds];
    cudaStream_t own_stream = nullptr;
    long long launches = 0;        // kernels issued by this handle (graph replays included)
    long long* launch_sink = nullptr;  // a binary32 shadow also counts into its handle's solver
    // Algorithmic bytes of those kernels: the values each must read and write
    // once (N = cells of the level, face arrays counted as N, s = value size).
    double alg_bytes = 0;
    double* bytes_sink = nullptr;
    long long newton_rejects = 0;  // Newton steps undone by the growth guard
    int report_not_converged = 0;  // GLIDE_TUNE_REPORT_NOT_CONVERGED
    bool last_not_converged = false;  // the last solve_loop ended short of its tolerances
    double last_relative = 0.0;
    int last_cycles = 0;

    // While set, the launches of the cycle bodies are appended here instead
    // of issued; launch sites that have no grouped form refuse.
    std::vector<RecOp>* rec = nullptr;

    template <class A>
    bool record(int op, int variant, dim3 g, const A& a, double bytes) {
        if (!rec) return false;
        RecOp r{op, variant, int(g.x), int(g.y), int(g.z), std::vector<unsigned char>(sizeof(A)), bytes};
        std::memcpy(r.args.data(), &a, sizeof(A));
        rec->push_back(std::move(r));
        return true;
    }

    // the staging maps of the launch just recorded
    template <int N>
    void attach_maps(const BoxMaps<N>& m) {
        const unsigned char* p = reinterpret_cast<const unsigned char*>(&m);
        rec->back().maps.assign(p, p + sizeof(m));
    }

    void not_recordable(const char* what) const {
        if (rec) fail(GLIDE_ERR_STATE, std::string(what) + " has no grouped form");
    }

    void counted(const char* what, double bytes) {
        check_launch(what);
        ++launches;
        if (launch_sink) ++*launch_sink;
        traffic(bytes);
    }

    // bytes moved without a kernel of ours (device-to-device copies)
    void traffic(double bytes) {
        alg_bytes += bytes;
        if (bytes_sink) *bytes_sink += bytes;
    }

    // `arrays` values per cell of level l
    double lb(int l, double arrays) const { return arrays * double(lv[l].ny) * double(lv[l].nx) * sizeof(R); }

    Solver(int ny, int nx, double dx, int L) {
        dtype = sizeof(R) == 8 ? GLIDE_F64 : GLIDE_F32;
        n_levels = L;
        fas[0] = default_fas();
        fas[1] = default_fas();
        fas[2] = default_tangent_fas();
        lv.resize(L);
        size_t bytes = 0;
        const size_t align = 256;
        for (int l = 0; l < L; ++l) {
            Level<R>& v = lv[l];
            v.ny = ny >> l;
            v.nx = nx >> l;
            v.dx = dx * double(1 << l);
            v.pu = round_up(v.nx + 1, 32);
            v.pv = round_up(v.nx, 32);
            v.pc = round_up(v.nx, 32);
            v.phys = default_phys();
            v.vk[0] = default_vanka();
            v.vk[1] = default_vanka();
            v.vk[2] = default_tangent_vanka();
            for (int f = 0; f < F_COUNT; ++f) {
                Kind k = field_kind(f);
                int rows = k == KV ? v.ny + 1 : v.ny;
                int cols = k == KU ? v.nx + 1 : v.nx;
                int pitch = k == KU ? v.pu : (k == KV ? v.pv : v.pc);
                v.a[f].rows = rows;
                v.a[f].cols = cols;
                v.a[f].pitch = pitch;
                v.a[f].p = reinterpret_cast<R*>(bytes);  // offset for now
                bytes += (size_t(rows) * pitch * sizeof(R) + align - 1) / align * align;
            }
        }
        const int nblk = lv[0].blocks_x() * lv[0].blocks_y();
        size_t partial_off = bytes;
        bytes += (size_t(nblk) * 3 * sizeof(double) + align - 1) / align * align;
        size_t norms_off = bytes;
        bytes += align;
        GCU(cudaMalloc(&arena, bytes));
        GCU(cudaMemset(arena, 0, bytes));
        for (auto& v : lv)
            for (int f = 0; f < F_COUNT; ++f)
                v.a[f].p = reinterpret_cast<R*>(arena + reinterpret_cast<size_t>(v.a[f].p));
        partial = reinterpret_cast<double*>(arena + partial_off);
        norms_dev = reinterpret_cast<double*>(arena + norms_off);
        err_dev = reinterpret_cast<int*>(arena + norms_off + 4 * sizeof(double));
        GCU(cudaMallocHost(&norms_host, 5 * sizeof(double)));
        // gamma holds thklim between sweep groups
        for (auto& v : lv) fill(v.a[GLIDE_GAMMA], R(v.phys.thklim), nullptr);
        GCU(cudaDeviceSynchronize());
    }

    ~Solver() override {
        for (CachedGraph& g : graphs)
            if (g.exec) cudaGraphExecDestroy(g.exec);
        for (R* b : blk) if (b) cudaFree(b);
        if (own_stream) cudaStreamDestroy(own_stream);
        if (norms_host) cudaFreeHost(norms_host);
        if (arena) cudaFree(arena);
    }

    // ---------------------------------------------------------- utilities
    static dim3 pw_grid(int rows, int cols) { return dim3((cols + 255) / 256, rows); }

    void fill(const Arr<R>& a, R val, cudaStream_t s) {
        if (record(G_FILL, 0, pw_grid(a.rows, a.cols), FillArgs<R>{a, val}, double(a.rows) * a.cols * sizeof(R)))
            return;
        k_fill<R><<<pw_grid(a.rows, a.cols), 256, 0, s>>>(a, val, a.rows, a.cols);
        counted("fill", double(a.rows) * a.cols * sizeof(R));
    }

    void copy(const Arr<R>& dst, const Arr<R>& src, cudaStream_t s) {
        if (record(G_COPY, 0, pw_grid(src.rows, src.cols), CopyArgs<R>{dst, src},
                   2.0 * src.rows * src.cols * sizeof(R)))
            return;
        GCU(cudaMemcpy2DAsync(dst.p, size_t(dst.pitch) * sizeof(R), src.p, size_t(src.pitch) * sizeof(R),
                              size_t(src.cols) * sizeof(R), src.rows, cudaMemcpyDeviceToDevice, s));
        traffic(2.0 * src.rows * src.cols * sizeof(R));
    }

    void restrict_field(int f, int l, cudaStream_t s, Arr<R> copy_to = Arr<R>()) {
        Level<R>& F = lv[l];
        Level<R>& C = lv[l + 1];
        restrict_arr(F.a[f], C.a[f], f == GLIDE_MASK ? kCellMax : -1, l, s, copy_to);
    }

    void restrict_arr(const Arr<R>& fa, const Arr<R>& ca, int cell_kind, int l, cudaStream_t s,
                      Arr<R> copy_to = Arr<R>()) {
        Level<R>& C = lv[l + 1];
        int kind;
        if (fa.cols == lv[l].nx + 1) kind = kFaceU;
        else if (fa.rows == lv[l].ny + 1) kind = kFaceV;
        else kind = cell_kind >= 0 ? cell_kind : kCellAvg;
        if (record(G_RESTRICT, 0, pw_grid(C.ny + 1, C.nx + 1), RestrictArgs<R>{fa, ca, copy_to, kind, C.ny, C.nx},
                   restrict_bytes(l, kind, copy_to.p != nullptr)))
            return;
        k_restrict<R><<<pw_grid(C.ny + 1, C.nx + 1), 256, 0, s>>>(fa, ca, copy_to, kind, C.ny, C.nx);
        counted("restrict", restrict_bytes(l, kind, copy_to.p != nullptr));
    }

    // one restriction into level l + 1: 2 fine faces or 4 fine cells read
    // per coarse value, the coarse value written (and its copy)
    double restrict_bytes(int l, int kind, bool copy) const {
        const double per = (kind == kFaceU || kind == kFaceV) ? 3.0 : 5.0;
        return lb(l + 1, per + (copy ? 1.0 : 0.0));
    }

    PhysR<R> physr(int l, double dt, bool freeze_calving) const {
        const Level<R>& v = lv[l];
        Phys p{v.phys.n, v.phys.eps_reg, v.phys.flotation_reg_driving, v.phys.m, v.phys.u_reg,
               v.phys.water_drag, v.phys.flotation_reg_sliding, v.phys.calving_rate,
               v.phys.flotation_reg_calving, v.phys.thklim};
        return PhysR<R>(p, v.dx, dt, freeze_calving ? 0.0 : v.phys.calving_rate);
    }

    void compute_phi(int l, double relax, cudaStream_t s) {
        Level<R>& v = lv[l];
        if (record(G_GROUNDED, 0, pw_grid(v.ny, v.nx),
                   GroundedArgs<R>{v.a[GLIDE_PHI], v.a[GLIDE_H], v.a[GLIDE_BED], R(v.phys.flotation_reg_driving),
                                   R(relax), v.ny, v.nx},
                   lb(l, 4)))
            return;
        k_grounded<R><<<pw_grid(v.ny, v.nx), 256, 0, s>>>(v.a[GLIDE_PHI], v.a[GLIDE_H], v.a[GLIDE_BED],
                                                          R(v.phys.flotation_reg_driving), R(relax), v.ny, v.nx);
        counted("grounded", lb(l, 4));  // H, bed, phi read; phi written
    }

    void set_rhs(int l, double dt, cudaStream_t s) {
        Level<R>& v = lv[l];
        const SetRhsArgs<R> a{v.a[GLIDE_F_H], v.a[GLIDE_H_PREV], v.a[GLIDE_SMB], R(dt), v.ny, v.nx};
        if (record(G_SET_RHS, 0, pw_grid(v.ny, v.nx), a, lb(l, 3))) return;
        k_set_rhs<R><<<pw_grid(v.ny, v.nx), 256, 0, s>>>(a);
        counted("set_rhs", lb(l, 3));
    }

    // residual into (o_*) = R(x) [- f] [- sub]; norms into norms_dev when asked
    void residual(int l, double dt, bool use_forcing, bool use_mask, bool freeze_calving, bool freeze_phi,
                  int out_u, int out_v, int out_H, const Arr<R>* sub, bool norms, cudaStream_t s,
                  bool active_set = false) {
        Level<R>& v = lv[l];
        if (!freeze_phi) compute_phi(l, 0.0, s);
        ResidualArgs<R> a;
        a.u = v.a[GLIDE_U]; a.v = v.a[GLIDE_V]; a.H = v.a[GLIDE_H];
        a.phi = v.a[GLIDE_PHI]; a.mask = v.a[GLIDE_MASK]; a.bed = v.a[GLIDE_BED]; a.B = v.a[GLIDE_B];
        a.beta = v.a[GLIDE_BETA]; a.gamma = v.a[GLIDE_GAMMA];
        a.f_u = v.a[GLIDE_F_U]; a.f_v = v.a[GLIDE_F_V]; a.f_H = v.a[GLIDE_F_H];
        a.o_u = v.a[out_u]; a.o_v = v.a[out_v]; a.o_H = v.a[out_H];
        if (sub) { a.s_u = sub[0]; a.s_v = sub[1]; a.s_H = sub[2]; }
        a.partial = norms ? partial : nullptr;
        a.err = err_dev;
        a.p = physr(l, dt, freeze_calving);
        a.ny = v.ny; a.nx = v.nx;
        a.use_forcing = use_forcing; a.use_mask = use_mask;
        a.active_set = active_set ? 1 : 0;
        dim3 g(v.blocks_x(), v.blocks_y());
        // u, v, H, phi, mask, bed, B, beta, gamma; forcing; subtrahend; 3 rows
        // written (and the active set)
        const double bytes = lb(l, 9 + (use_forcing ? 3 : 0) + (sub ? 3 : 0) + 3 + (active_set ? 1 : 0));
        if (record(G_RESIDUAL, 0, g, a, bytes)) {
            attach_maps(box_maps(l, kStateBoxes));
        } else {
            k_residual<R><<<g, 256, 0, s>>>(a, box_maps(l, kStateBoxes));
            counted("residual", bytes);
        }
        if (norms) finish_norms(int(g.x * g.y), s);
    }

    // the norm vector of the per-block partials of the last stencil pass
    void finish_norms(int nblocks, cudaStream_t s) {
        const double bytes = 24.0 * nblocks + 32.0;
        if (record(G_NORMS, 0, dim3(1), NormsArgs{partial, nblocks, norms_dev}, bytes)) return;
        k_finish_norms<<<1, kNormThreads, 0, s>>>(partial, nblocks, norms_dev);
        counted("finish_norms", bytes);
    }

    void vanka_dump(int l, double dt, R* J, R* r, cudaStream_t s) {
        Level<R>& v = lv[l];
        ResidualArgs<R> a;
        a.u = v.a[GLIDE_U]; a.v = v.a[GLIDE_V]; a.H = v.a[GLIDE_H];
        a.phi = v.a[GLIDE_PHI]; a.mask = v.a[GLIDE_MASK]; a.bed = v.a[GLIDE_BED]; a.B = v.a[GLIDE_B];
        a.beta = v.a[GLIDE_BETA]; a.gamma = v.a[GLIDE_GAMMA];
        a.f_u = v.a[GLIDE_F_U]; a.f_v = v.a[GLIDE_F_V]; a.f_H = v.a[GLIDE_F_H];
        a.partial = nullptr;
        a.err = err_dev;
        a.p = physr(l, dt, false);
        a.ny = v.ny; a.nx = v.nx;
        a.use_forcing = 1; a.use_mask = 0; a.active_set = 0;
        not_recordable("vanka_dump");
        k_vanka_dump<R><<<dim3(v.blocks_x(), v.blocks_y()), 256, 0, s>>>(a, J, r);
        counted("vanka_dump", lb(l, 11 + 30));
    }

    // the norm vector and, in the same copy, the error word behind it
    void read_norms(double out[4], cudaStream_t s) {
        not_recordable("read_norms");
        GCU(cudaMemcpyAsync(norms_host, norms_dev, 4 * sizeof(double) + sizeof(int), cudaMemcpyDeviceToHost, s));
        GCU(cudaStreamSynchronize(s));
        for (int q = 0; q < 4; ++q) out[q] = norms_host[q];
        int e;
        std::memcpy(&e, norms_host + 4, sizeof(int));
        if (e) {
            // clear the word, so the next call on this handle starts clean
            GCU(cudaMemsetAsync(err_dev, 0, sizeof(int), s));
            GCU(cudaStreamSynchronize(s));
            if (e & kStageBadMaps) fail(GLIDE_ERR_STATE, "a kernel's staging maps failed their check");
            fail(GLIDE_ERR_TIMEOUT, "a kernel's bounded wait for its tile copies gave up");
        }
    }

    // TMA staging needs a level at least one box wide and high
    bool tma_level(int l, int bh = kBoxH) const { return use_tma && lv[l].nx >= kBoxW && lv[l].ny >= bh; }

    const CUtensorMap& tmap(int l, int f, int bh = kBoxH) {
        int w = 0;
        while (w < 3 && kTmaHeights[w] != bh) ++w;
        if (w == 3) fail(GLIDE_ERR_STATE, "no tensor-map slot for this box height");
        if (tmaps[w].empty()) {
            tmaps[w].resize(size_t(n_levels) * F_COUNT);
            tmap_done[w].assign(size_t(n_levels) * F_COUNT, 0);
        }
        const size_t k = size_t(l) * F_COUNT + f;
        if (!tmap_done[w][k]) {
            PFN_cuTensorMapEncodeTiled_v12000 enc = tensor_map_encoder();
            if (!enc) fail(GLIDE_ERR_CUDA, "cuTensorMapEncodeTiled is not available from the driver");
            const Arr<R>& a = lv[l].a[f];
            const cuuint64_t dims[2] = {cuuint64_t(a.cols), cuuint64_t(a.rows)};
            const cuuint64_t strides[1] = {cuuint64_t(a.pitch) * sizeof(R)};
            const cuuint32_t box[2] = {cuuint32_t(kBoxW), cuuint32_t(bh)};
            const cuuint32_t estr[2] = {1, 1};
            const CUresult r = enc(&tmaps[w][k], sizeof(R) == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64
                                                                  : CU_TENSOR_MAP_DATA_TYPE_FLOAT32,
                                   2, a.p, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                                   CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                                   CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
            if (r != CUDA_SUCCESS) fail(GLIDE_ERR_CUDA, "cuTensorMapEncodeTiled failed");
            tmap_done[w][k] = 1;
        }
        return tmaps[w][k];
    }

    template <int N>
    BoxMaps<N> box_maps(int l, const int (&fields)[N], int bh = kBoxH) {
        BoxMaps<N> m;
        m.use = tma_level(l, bh) ? 1 : 0;
        m.wait_polls = tma_wait_polls;
        if (m.use)
            for (int q = 0; q < N; ++q) m.m[q] = tmap(l, fields[q], bh);
        return m;
    }

    // n additive-Vanka sweeps on level l, ending in the home state buffers
    void sweeps(int l, double dt, int n, int gmode, bool freeze_calving, bool freeze_phi, int* iters,
                cudaStream_t s) {
        if (n <= 0) return;
        Level<R>& v = lv[l];
        const glide_vanka_config& c = v.vk[0];
        const bool phi_live = !freeze_phi && c.relax_phi == 0.0;
        const int start_alt = n & 1;
        if (start_alt) {
            copy(v.a[F_U_ALT], v.a[GLIDE_U], s);
            copy(v.a[F_V_ALT], v.a[GLIDE_V], s);
            copy(v.a[F_H_ALT], v.a[GLIDE_H], s);
        }
        SweepArgs<R> a;
        a.phi = v.a[GLIDE_PHI]; a.mask = v.a[GLIDE_MASK]; a.bed = v.a[GLIDE_BED]; a.B = v.a[GLIDE_B];
        a.beta = v.a[GLIDE_BETA];
        a.f_u = v.a[GLIDE_F_U]; a.f_v = v.a[GLIDE_F_V]; a.f_H = v.a[GLIDE_F_H];
        a.gamma = v.a[GLIDE_GAMMA];
        a.wH = v.a[F_W_H]; a.chi = v.a[F_CHI];
        a.chi_c = (l + 1 < n_levels) ? lv[l + 1].a[F_CHI] : Arr<R>();
        a.p = physr(l, dt, freeze_calving);
        a.omega = R(c.omega); a.ssa_damping = R(c.ssa_damping); a.mc_damping = R(c.mc_damping);
        // reference mode: the kernel's fixed 0.5 (vanka.cu:615); otherwise the configured value
        a.relax = quirks ? R(0.5) : R(c.relaxation);
        a.newton_steps = c.newton_steps;
        a.ny = v.ny; a.nx = v.nx;
        dim3 g(v.blocks_x(), v.blocks_y());
        for (int k = 0; k < n; ++k) {
            const bool in_alt = (start_alt ^ (k & 1)) != 0;
            const int U0 = GLIDE_U, V0 = GLIDE_V, H0 = GLIDE_H, U1 = F_U_ALT, V1 = F_V_ALT, H1 = F_H_ALT;
            const int iu = in_alt ? U1 : U0, iv = in_alt ? V1 : V0, ih = in_alt ? H1 : H0;
            const int ou = in_alt ? U0 : U1, ov = in_alt ? V0 : V1, oh = in_alt ? H0 : H1;
            a.u = v.a[iu]; a.v = v.a[iv]; a.H = v.a[ih];
            a.uo = v.a[ou]; a.vo = v.a[ov]; a.Ho = v.a[oh];
            a.iters = (k == n - 1) ? iters : nullptr;
            if (!freeze_phi && !phi_live) {
                const GroundedArgs<R> ga{v.a[GLIDE_PHI], v.a[ih], v.a[GLIDE_BED], R(v.phys.flotation_reg_driving),
                                         R(c.relax_phi), v.ny, v.nx};
                if (!record(G_GROUNDED, 0, pw_grid(v.ny, v.nx), ga, lb(l, 4))) {
                    k_grounded<R><<<pw_grid(v.ny, v.nx), 256, 0, s>>>(ga.phi, ga.H, ga.bed, ga.c, ga.relax, v.ny,
                                                                      v.nx);
                    counted("grounded", lb(l, 4));
                }
            }
            launch_sweep(a, gmode, phi_live, g, s, lb(l, 15));
        }
    }

    template <int MINB>
    void launch_sweep_occ(const SweepArgs<R>& a, int gmode, bool phi_live, dim3 g, cudaStream_t s) {
#define GLIDE_SWEEP(GM, PL) k_vanka_sweep<R, GM, PL, MINB><<<g, kSweepThreads, 0, s>>>(a)
        if (gmode == kGammaArray) { if (phi_live) GLIDE_SWEEP(kGammaArray, true); else GLIDE_SWEEP(kGammaArray, false); }
        else if (gmode == kGammaWChi) { if (phi_live) GLIDE_SWEEP(kGammaWChi, true); else GLIDE_SWEEP(kGammaWChi, false); }
        else { if (phi_live) GLIDE_SWEEP(kGammaWPhi, true); else GLIDE_SWEEP(kGammaWPhi, false); }
#undef GLIDE_SWEEP
    }

    // one fused sweep: u, v, H, f_u, f_v, f_H, bed, B, beta, gamma, phi read;
    // u, v, H, mask written (15 N s)
    void launch_sweep(const SweepArgs<R>& a, int gmode, bool phi_live, dim3 g, cudaStream_t s, double bytes) {
        if (rec) {
            SweepArgs<R> ga = a;
            ga.gmode = gmode;
            record(G_SWEEP, (phi_live ? 1 : 0) | (sweep_blocks_per_sm >= 2 ? 2 : 0), g, ga, bytes);
            return;
        }
        if (sweep_blocks_per_sm >= 2) launch_sweep_occ<2>(a, gmode, phi_live, g, s);
        else launch_sweep_occ<1>(a, gmode, phi_live, g, s);
        counted("vanka_sweep", bytes);
    }

    // Restrictions of several fields of level l in one launch; each job is
    // (field, field receiving a copy of the coarse values or -1, cell kind
    // or -1 for the field's own kind).
    struct RJob { int f, copy_to, cell_kind; };
    void restrict_batch(int l, const RJob* jobs, int n, cudaStream_t s) {
        Level<R>& F = lv[l];
        Level<R>& C = lv[l + 1];
        RestrictJobs<R> b;
        if (n > kMaxRestrictJobs) fail(GLIDE_ERR_STATE, "too many restrictions in one batch");
        for (int q = 0; q < n; ++q) {
            const Arr<R>& fa = F.a[jobs[q].f];
            b.f[q] = fa;
            b.c[q] = C.a[jobs[q].f];
            b.copy[q] = jobs[q].copy_to >= 0 ? C.a[jobs[q].copy_to] : Arr<R>();
            if (fa.cols == F.nx + 1) b.kind[q] = kFaceU;
            else if (fa.rows == F.ny + 1) b.kind[q] = kFaceV;
            else b.kind[q] = jobs[q].cell_kind >= 0 ? jobs[q].cell_kind
                                                    : (jobs[q].f == GLIDE_MASK ? kCellMax : kCellAvg);
        }
        b.nyc = C.ny; b.nxc = C.nx;
        dim3 g = pw_grid(C.ny + 1, C.nx + 1);
        g.z = n;
        double bytes = 0;
        for (int q = 0; q < n; ++q) bytes += restrict_bytes(l, b.kind[q], jobs[q].copy_to >= 0);
        if (record(G_RESTRICT_BATCH, 0, g, b, bytes)) return;
        k_restrict_batch<R><<<g, 256, 0, s>>>(b);
        counted("restrict_batch", bytes);
    }

    // the u, v and H corrections of level l (fields x, snapshots w, kinds k)
    void correct3(int l, const int (&x)[3], const int (&w)[3], const int (&kinds)[3], int mode, cudaStream_t s) {
        Level<R>& F = lv[l];
        Level<R>& C = lv[l + 1];
        CorrectJobs<R> b;
        for (int q = 0; q < 3; ++q) {
            CorrectArgs<R>& a = b.j[q];
            a.x = F.a[x[q]]; a.w = F.a[w[q]]; a.xc = C.a[x[q]]; a.wc = C.a[w[q]];
            a.kind = kinds[q]; a.mode = mode; a.vquirk = quirks; a.nyf = F.ny; a.nxf = F.nx;
        }
        dim3 g = pw_grid(F.ny + 1, F.nx + 1);
        g.z = 3;
        // per field: fine x and w read, x written; coarse x and w read
        const double bytes = 3 * (lb(l, 3) + lb(l + 1, 2));
        if (record(G_CORRECT_BATCH, 0, g, b, bytes)) return;
        k_correct_batch<R><<<g, 256, 0, s>>>(b);
        counted("correct_batch", bytes);
    }


    // ------------------------------------------------------ FASCD V-cycle
    // glide/multigrid.py:536-645
    void vcycle(int l, bool finest, double dt, cudaStream_t s) {
        const glide_fas_config& c = fas[0];
        const bool coarse = !finest;
        const bool fcal = coarse && c.freeze_coarse_calving, fphi = coarse && c.freeze_coarse_phi;
        Level<R>& v = lv[l];
        if (finest) {
            const SnapshotArgs<R> sa{v.a[GLIDE_U], v.a[GLIDE_V], v.a[GLIDE_H], v.a[F_W_U], v.a[F_W_V],
                                     v.a[F_W_H], v.a[F_CHI], R(v.phys.thklim), v.ny, v.nx};
            // u, v, H read; w_u, w_v, w_H, chi written
            if (!record(G_SNAPSHOT, 0, pw_grid(v.ny + 1, v.nx + 1), sa, lb(l, 7))) {
                k_snapshot<R><<<pw_grid(v.ny + 1, v.nx + 1), 256, 0, s>>>(sa);
                counted("snapshot", lb(l, 7));
            }
        }
        if (l == n_levels - 1) {
            sweeps(l, dt, c.coarsest_steps, kGammaWChi, fcal, fphi, nullptr, s);
            return;
        }
        Level<R>& n = lv[l + 1];
        restrict_arr(v.a[F_CHI], n.a[F_CHI], kCellMax, l, s);
        sweeps(l, dt, c.pre_steps, kGammaWPhi, fcal, fphi, nullptr, s);
        // the residual (phi frozen) reads level l only, so the state and the
        // residual are restricted together after it, in one launch
        residual(l, dt, true, false, fcal, true, GLIDE_R_U, GLIDE_R_V, GLIDE_R_H, nullptr, false, s);
        {
            const RJob jobs[9] = {{GLIDE_U, F_W_U, -1}, {GLIDE_V, F_W_V, -1}, {GLIDE_H, F_W_H, -1},
                                  {GLIDE_H_PREV, -1, -1}, {GLIDE_PHI, -1, -1}, {GLIDE_MASK, -1, -1},
                                  {GLIDE_R_U, -1, -1}, {GLIDE_R_V, -1, -1}, {GLIDE_R_H, -1, -1}};
            restrict_batch(l, jobs, 9, s);
        }
        const Arr<R> sub[3] = {n.a[GLIDE_R_U], n.a[GLIDE_R_V], n.a[GLIDE_R_H]};
        residual(l + 1, dt, false, false, c.freeze_coarse_calving != 0, c.freeze_coarse_phi != 0, GLIDE_F_U,
                 GLIDE_F_V, GLIDE_F_H, sub, false, s);
        vcycle(l + 1, false, dt, s);
        correct3(l, {GLIDE_U, GLIDE_V, GLIDE_H}, {F_W_U, F_W_V, F_W_H}, {kFaceU, kFaceV, kCellAvg}, 0, s);
        sweeps(l, dt, c.post_steps, kGammaWChi, fcal, fphi, nullptr, s);
        if (finest) sweeps(l, dt, c.finest_steps, kGammaArray, false, false, nullptr, s);
    }

    void check_quirks() {
        if (quirks)
            for (int l = 0; l + 1 < n_levels; ++l)
                if (lv[l].ny != lv[l].nx)
                    fail(GLIDE_ERR_SHAPE, "reference-quirk v prolongation needs square levels (ny == nx)");
    }

    // Replay (or capture) one V-cycle followed by the convergence residual.
    void cycle_and_check(int kind, int start, double dt, cudaStream_t s) {
        auto body = [&]() {
            if (kind == 0) {
                vcycle(start, true, dt, s);
                residual(start, dt, true, true, false, true, GLIDE_R_U, GLIDE_R_V, GLIDE_R_H, nullptr, true, s);
            } else if (kind == 1) {
                adj_vcycle(start, true, dt, s);
                adj_residual(start, dt, true, s);
            } else {
                if (kind == 4) {
                    newton_cycle(start, dt, s);
                } else if constexpr (sizeof(R) == 8) {
                    if (kind == 2) mixed_cycle(start, dt, s);
                    else mixed_adj_cycle(start, dt, s);
                }
            }
        };
        if (!use_graphs) {
            body();
            return;
        }
        // The legacy default stream cannot be captured.  A stream created with
        // default (blocking) flags is ordered against it implicitly, so the
        // graph runs there when the caller passed NULL.
        if (s == nullptr) {
            if (!own_stream) GCU(cudaStreamCreate(&own_stream));
            s = own_stream;
        }
        CachedGraph& cg = graphs[kind];
        if (!cg.exec || cg.version != version || cg.dt != dt || cg.start != start) {
            if (cg.exec) { cudaGraphExecDestroy(cg.exec); cg.exec = nullptr; }
            std::lock_guard<std::mutex> lock(g_capture_mu);
            cudaGraph_t g;
            const long long before = launches;
            const double bytes_before = alg_bytes;
            GCU(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
            try {
                body();
            } catch (...) {
                cudaStreamEndCapture(s, &g);
                if (g) cudaGraphDestroy(g);
                launches = before;
                alg_bytes = bytes_before;
                throw;
            }
            cg.launches = launches - before;
            cg.bytes = alg_bytes - bytes_before;
            launches = before;
            alg_bytes = bytes_before;
            GCU(cudaStreamEndCapture(s, &g));
            cudaError_t e = cudaGraphInstantiate(&cg.exec, g, 0);
            cudaGraphDestroy(g);
            if (e != cudaSuccess) fail(GLIDE_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(e));
            cg.version = version; cg.dt = dt; cg.start = start;
        }
        GCU(cudaGraphLaunch(cg.exec, s));
        launches += cg.launches;
        alg_bytes += cg.bytes;
    }

    // ------------------------------------------------ mixed precision
    // binary64 state and residual on the solve level; a binary32 shadow
    // hierarchy runs the smoother and every coarse level.  Each outer step is
    // a nonlinear defect correction:
    //   r = R64(x)  (unmasked),   g = F32(fl(x)) - fl(r),
    //   y = FASCD V-cycle(s) of F32(y) = g from y0 = fl(x),
    //   x <- x + (y - fl(x))  (binary64),  mask <- mask32, H = gamma on masked cells,
    // and the convergence test is the reference's masked binary64 residual.
    std::unique_ptr<Solver<float>> lo;
    int mixed_inner = 1;

    template <class D, class Src>
    void convert(const Arr<D>& d, const Arr<Src>& src, double scale, cudaStream_t s) {
        not_recordable("convert");
        k_convert<D, Src><<<pw_grid(src.rows, src.cols), 256, 0, s>>>(d, src, scale, src.rows, src.cols);
        counted("convert", double(src.rows) * src.cols * (sizeof(D) + sizeof(Src)));
    }

    void sync_shadow() {
        Solver<float>& f = *lo;
        for (int q = 0; q < 3; ++q) f.fas[q] = fas[q];
        f.quirks = quirks;
        f.sweep_blocks_per_sm = sweep_blocks_per_sm;
        f.use_graphs = 0;
        f.use_tma = use_tma;
        f.tma_wait_polls = tma_wait_polls;
        f.err_dev = err_dev;  // shadow kernels report into this handle's error word
        f.launch_sink = &launches;  // and count into its launches (captured cycles included)
        f.bytes_sink = &alg_bytes;
        for (int l = 0; l < n_levels; ++l) {
            if (f.lv[l].phys.thklim != lv[l].phys.thklim)
                f.fill(f.lv[l].a[GLIDE_GAMMA], float(lv[l].phys.thklim), nullptr);
            f.lv[l].phys = lv[l].phys;
            for (int q = 0; q < 3; ++q) f.lv[l].vk[q] = lv[l].vk[q];
        }
    }

    // binary64 level-l fields -> shadow, then restricted down in the shadow
    void push_to_shadow(int l, std::initializer_list<int> fields, bool restrict_down, cudaStream_t s) {
        Solver<float>& f = *lo;
        for (int fld : fields) {
            convert(f.lv[l].a[fld], lv[l].a[fld], 1.0, s);
            if (restrict_down)
                for (int q = l; q + 1 < n_levels; ++q) f.restrict_field(fld, q, s);
        }
    }

    void mixed_cycle(int l, double dt, cudaStream_t s) {
        Solver<float>& f = *lo;
        Level<R>& D = lv[l];
        Level<float>& F = f.lv[l];
        not_recordable("mixed_cycle");
        push_to_shadow(l, {GLIDE_U, GLIDE_V, GLIDE_H, GLIDE_MASK, GLIDE_PHI}, false, s);
        residual(l, dt, true, false, false, true, GLIDE_R_U, GLIDE_R_V, GLIDE_R_H, nullptr, false, s);
        push_to_shadow(l, {GLIDE_R_U, GLIDE_R_V, GLIDE_R_H}, false, s);
        const Arr<float> sub[3] = {F.a[GLIDE_R_U], F.a[GLIDE_R_V], F.a[GLIDE_R_H]};
        f.residual(l, dt, false, false, false, true, GLIDE_F_U, GLIDE_F_V, GLIDE_F_H, sub, false, s);
        for (int k = 0; k < mixed_inner; ++k) f.vcycle(l, true, dt, s);
        k_defect_update<R, float><<<pw_grid(D.ny + 1, D.nx + 1), 256, 0, s>>>(
            D.a[GLIDE_U], D.a[GLIDE_V], D.a[GLIDE_H], D.a[GLIDE_MASK], D.a[GLIDE_GAMMA], F.a[GLIDE_U],
            F.a[GLIDE_V], F.a[GLIDE_H], F.a[GLIDE_MASK], D.ny, D.nx);
        // binary64 u, v, H, mask, gamma read and u, v, H, mask written;
        // binary32 u, v, H, mask read
        counted("defect_update", lb(l, 9) + double(D.ny) * D.nx * 4 * sizeof(float));
        residual(l, dt, true, true, false, false, GLIDE_R_U, GLIDE_R_V, GLIDE_R_H, nullptr, true, s);
    }

    void mixed_adj_cycle(int l, double dt, cudaStream_t s) {
        Solver<float>& f = *lo;
        Level<R>& D = lv[l];
        Level<float>& F = f.lv[l];
        adj_residual(l, dt, false, s);
        for (int fld : {GLIDE_LAMBDA_U, GLIDE_LAMBDA_V, GLIDE_LAMBDA_H}) f.fill(F.a[fld], 0.0f, s);
        convert(F.a[GLIDE_ADJ_F_U], D.a[GLIDE_ADJ_R_U], -1.0, s);
        convert(F.a[GLIDE_ADJ_F_V], D.a[GLIDE_ADJ_R_V], -1.0, s);
        convert(F.a[GLIDE_ADJ_F_H], D.a[GLIDE_ADJ_R_H], -1.0, s);
        for (int k = 0; k < mixed_inner; ++k) f.adj_vcycle(l, true, dt, s);
        convert_add(D.a[GLIDE_LAMBDA_U], F.a[GLIDE_LAMBDA_U], s);
        convert_add(D.a[GLIDE_LAMBDA_V], F.a[GLIDE_LAMBDA_V], s);
        convert_add(D.a[GLIDE_LAMBDA_H], F.a[GLIDE_LAMBDA_H], s);
        adj_residual(l, dt, true, s);
    }

    template <class Src>
    void convert_add(const Arr<R>& d, const Arr<Src>& src, cudaStream_t s) {
        not_recordable("convert_add");
        k_add_converted<R, Src><<<pw_grid(src.rows, src.cols), 256, 0, s>>>(d, src, src.rows, src.cols);
        counted("add_converted", double(src.rows) * src.cols * (2 * sizeof(R) + sizeof(Src)));
    }

    void forward_mixed(double dt, int start, glide_stats* st, cudaStream_t s) {
        sync_shadow();
        lo->check_quirks();
        set_rhs(start, dt, s);
        push_to_shadow(start, {GLIDE_BED, GLIDE_B, GLIDE_BETA, GLIDE_SMB, GLIDE_H_PREV}, true, s);
        residual(start, dt, true, true, false, false, GLIDE_R_U, GLIDE_R_V, GLIDE_R_H, nullptr, true, s);
        double nr[4];
        read_norms(nr, s);
        solve_loop(2, start, dt, nr, st, s);
    }

    void backward_mixed(double dt, int start, int grad_mask, glide_stats* st, cudaStream_t s) {
        sync_shadow();
        lo->check_quirks();
        push_to_shadow(start, {GLIDE_BED, GLIDE_B, GLIDE_BETA, GLIDE_SMB}, true, s);
        push_to_shadow(start, {GLIDE_U, GLIDE_V, GLIDE_H, GLIDE_H_PREV, GLIDE_PHI, GLIDE_MASK}, false, s);
        adj_residual(start, dt, true, s);
        double nr[4];
        read_norms(nr, s);
        solve_loop(3, start, dt, nr, st, s);
        gradients(start, dt, grad_mask, s);
    }

    void forward(double dt, int start, glide_stats* st, cudaStream_t s) {
        check_level(start);
        check_quirks();
        if (forward_method == 1) ensure_blocks();
        if constexpr (sizeof(R) == 8) {
            if (lo) lo->ensure_blocks();
        }
        if constexpr (sizeof(R) == 8) {
            if (lo) {
                forward_mixed(dt, start, st, s);
                return;
            }
        }
        set_rhs(start, dt, s);
        residual(start, dt, true, true, false, false, GLIDE_R_U, GLIDE_R_V, GLIDE_R_H, nullptr, true, s);
        double nr[4];
        read_norms(nr, s);
        solve_loop(0, start, dt, nr, st, s);
    }

    void solve_loop(int kind, int start, double dt, double nr[4], glide_stats* st, cudaStream_t s) {
        const glide_fas_config& c = fas[kind & 1];  // 0/2 forward, 1/3 adjoint
        const double r0 = nr[3];
        if (!std::isfinite(r0)) fail(GLIDE_ERR_NONFINITE, "initial residual norm is not finite");
        double rel = 1.0, ab = r0;
        int it = 0;
        bool in_newton = false;
        if (st) {
            std::memset(st, 0, sizeof(*st));
            st->initial_norm = r0;
            st->history[0] = r0;
        }
        // Newton guards.  Each Newton step starts from a saved state; a step
        // whose residual grows (or is not finite) is undone, and Newton waits
        // until FASCD has cut the residual another tenfold.  Two consecutive
        // steps that fail to cut it by `newton_stall_ratio` hand the rest of
        // the solve back to FASCD.  On a mixed handle the FASCD cycles after
        // the switch run in binary64: the binary32 defect correction stops near
        // the binary32 rounding level of the residual.
        bool newton_off = false;
        int stall = 0;
        double gate = newton_switch;
        double prev = ab;
        Level<R>& L0 = lv[start];
        while (rel > c.relative_tolerance && ab > c.absolute_tolerance && it < c.maximum_vcycles) {
            // forward solves may finish with Newton steps once the FAS phase is close
            int k = kind;
            const bool forward_newton = (kind == 0 || kind == 2) && forward_method == 1;
            const bool newton_phase = forward_newton && rel <= newton_switch;
            if (newton_phase && !newton_off && rel <= gate) k = 4;
            else if (newton_phase && kind == 2) k = 0;
            if (k == 4 && !in_newton) {
                // the Newton residual (active set decided inline) of the
                // current state: the norm the first step is judged against
                newton_prologue(start, dt, true, s);
                read_norms(nr, s);
                prev = nr[3];
                in_newton = true;
            }
            if (k != 4) in_newton = false;
            if (k == 4) {
                copy(L0.a[F_BK_U], L0.a[GLIDE_U], s);
                copy(L0.a[F_BK_V], L0.a[GLIDE_V], s);
                copy(L0.a[F_BK_H], L0.a[GLIDE_H], s);
                copy(L0.a[F_BK_MASK], L0.a[GLIDE_MASK], s);
            }
            cycle_and_check(k, start, dt, s);
            read_norms(nr, s);
            ab = nr[3];
            if (k == 4 && !(ab <= prev)) {  // grew or not finite: undo the step
                copy(L0.a[GLIDE_U], L0.a[F_BK_U], s);
                copy(L0.a[GLIDE_V], L0.a[F_BK_V], s);
                copy(L0.a[GLIDE_H], L0.a[F_BK_H], s);
                copy(L0.a[GLIDE_MASK], L0.a[F_BK_MASK], s);
                ab = prev;
                gate = 0.1 * (prev / r0);
                in_newton = false;
                stall = 0;
                ++newton_rejects;
            }
            if (!std::isfinite(ab)) fail(GLIDE_ERR_NONFINITE, "residual norm became non-finite");
            rel = ab / r0;
            if (k == 4 && in_newton) {
                stall = ab > newton_stall_ratio * prev ? stall + 1 : 0;
                if (stall >= 2) newton_off = true;
            }
            prev = ab;
            ++it;
            if (st && it < GLIDE_MAX_HISTORY) st->history[it] = ab;
        }
        if (st) {
            st->vcycles = it;
            st->final_norm = ab;
            for (int q = 0; q < 3; ++q) st->norms[q] = nr[q];
        }
        last_not_converged = !(rel <= c.relative_tolerance || ab <= c.absolute_tolerance);
        last_relative = rel;
        last_cycles = it;
    }

    // after a whole forward / backward call: the optional status of a solve
    // that stopped at the cycle cap
    void report_convergence() const {
        if (report_not_converged && last_not_converged)
            fail(GLIDE_ERR_NOT_CONVERGED, "solve stopped after " + std::to_string(last_cycles) +
                                              " cycles at relative residual " + std::to_string(last_relative));
    }

    void check_level(int l) const {
        if (l < 0 || l >= n_levels) fail(GLIDE_ERR_ARG, "level out of range");
    }

    // ------------------------------------------------------ linear systems
    // The adjoint J^T lambda = f (FASAdjoint, glide/multigrid.py:857-973) and
    // the tangent J e = f of the Newton outer iteration share one linear
    // multigrid: the same transfers, block smoother and V-cycle, with the
    // operator transposed or not.
    struct Lin {
        int x[3], f[3], r[3], w[3];
        bool tr;  // transpose: the adjoint system
        int cfg;  // schedule / smoother config: 1 adjoint, 2 tangent
    };
    static Lin adj_sys() {
        return {{GLIDE_LAMBDA_U, GLIDE_LAMBDA_V, GLIDE_LAMBDA_H}, {GLIDE_ADJ_F_U, GLIDE_ADJ_F_V, GLIDE_ADJ_F_H},
                {GLIDE_ADJ_R_U, GLIDE_ADJ_R_V, GLIDE_ADJ_R_H}, {F_WL_U, F_WL_V, F_WL_H}, true, 1};
    }
    static Lin tan_sys() {
        return {{F_E_U, F_E_V, F_E_H}, {F_TF_U, F_TF_V, F_TF_H}, {F_TR_U, F_TR_V, F_TR_H},
                {F_TW_U, F_TW_V, F_TW_H}, false, 2};
    }

    // out = Op(x) [- f] [- sub], Op = J^T (vjp) or J (jvp) at the level's state
    // jvp_flags (the JVP only): GLIDE_USE_MASK and GLIDE_FREEZE_CALVING as in
    // glide_jvp; the solver's own tangent operator keeps the mask and calving.
    void lin_op(int l, double dt, const Lin& L, const int* out, const int* sub, bool use_forcing, bool norms,
                bool ref_rows, cudaStream_t s, int jvp_flags = GLIDE_USE_MASK) {
        Level<R>& v = lv[l];
        VjpArgs<R> a;
        a.u = v.a[GLIDE_U]; a.v = v.a[GLIDE_V]; a.H = v.a[GLIDE_H];
        a.phi = v.a[GLIDE_PHI]; a.mask = v.a[GLIDE_MASK]; a.bed = v.a[GLIDE_BED]; a.B = v.a[GLIDE_B];
        a.beta = v.a[GLIDE_BETA];
        a.lu = v.a[L.x[0]]; a.lv = v.a[L.x[1]]; a.lH = v.a[L.x[2]];
        a.f_u = v.a[L.f[0]]; a.f_v = v.a[L.f[1]]; a.f_H = v.a[L.f[2]];
        a.o_u = v.a[out[0]]; a.o_v = v.a[out[1]]; a.o_H = v.a[out[2]];
        if (sub) { a.s_u = v.a[sub[0]]; a.s_v = v.a[sub[1]]; a.s_H = v.a[sub[2]]; }
        a.partial = norms ? partial : nullptr;
        a.err = err_dev;
        a.p = physr(l, dt, !L.tr && (jvp_flags & GLIDE_FREEZE_CALVING));
        a.ny = v.ny; a.nx = v.nx; a.use_forcing = use_forcing;
        dim3 g((a.nx + kTileA - 1) / kTileA, (a.ny + kTileA - 1) / kTileA);
        // u, v, H, phi, mask, bed, beta, B and the three unknowns read, the
        // forcing and the subtrahend when given, three rows written
        const double lin_bytes = lb(l, 11 + (use_forcing ? 3 : 0) + (sub ? 3 : 0) + 3);
        if (L.tr) {
            const int fl[AdjTile<R>::NB] = {GLIDE_U, GLIDE_V, GLIDE_H, GLIDE_PHI, GLIDE_BED, GLIDE_BETA,
                                            GLIDE_B, L.x[0], L.x[1]};
            if (record(G_VJP, 0, g, a, lin_bytes)) {
                attach_maps(box_maps(l, fl, AdjTile<R>::BH));
            } else {
                k_vjp<R><<<g, kTileA * kTileA, 0, s>>>(a, box_maps(l, fl, AdjTile<R>::BH));
                counted("vjp", lin_bytes);
            }
        } else {
            const int fl[JvpTile<R>::NB] = {GLIDE_U, GLIDE_V, L.x[0], L.x[1], GLIDE_H, GLIDE_PHI, GLIDE_BED,
                                            GLIDE_BETA, GLIDE_B, L.x[2]};
            const int mode = (ref_rows ? 1 : 0) | ((jvp_flags & GLIDE_USE_MASK) ? 0 : 2);
            if (record(G_JVP, 0, g, JvpOpArgs<R>{a, mode}, lin_bytes)) {
                attach_maps(box_maps(l, fl));
            } else {
                k_jvp<R><<<g, kTileA * kTileA, 0, s>>>(a, mode, box_maps(l, fl));
                counted("jvp", lin_bytes);
            }
        }
        if (norms) finish_norms(int(g.x * g.y), s);
    }

    void vjp_into(int l, double dt, bool use_forcing, int ou, int ov, int oh, cudaStream_t s) {
        const int out[3] = {ou, ov, oh};
        lin_op(l, dt, adj_sys(), out, nullptr, use_forcing, false, false, s);
    }

    void lin_residual(int l, double dt, const Lin& L, bool norms, cudaStream_t s) {
        lin_op(l, dt, L, L.r, nullptr, true, norms, false, s);
    }

    void adj_residual(int l, double dt, bool norms, cudaStream_t s) { lin_residual(l, dt, adj_sys(), norms, s); }

    // stored block factors of the linear smoother, one buffer per level
    std::vector<R*> blk;

    // allocated on first use, before any stream capture begins
    void ensure_blocks() {
        if (!blk.empty()) return;
        std::lock_guard<std::mutex> lock(g_capture_mu);
        blk.assign(n_levels, nullptr);
        for (int l = 0; l < n_levels; ++l)
            GCU(cudaMalloc(&blk[l], size_t(25) * lv[l].ny * lv[l].pc * sizeof(R)));
    }

    BlockArgs<R> block_args(int l, double dt, const Lin& L) {
        Level<R>& v = lv[l];
        if (blk.empty()) fail(GLIDE_ERR_STATE, "block factor buffers not allocated");
        const glide_vanka_config& c = v.vk[L.cfg];
        BlockArgs<R> a;
        a.u = v.a[GLIDE_U]; a.v = v.a[GLIDE_V]; a.H = v.a[GLIDE_H];
        a.phi = v.a[GLIDE_PHI]; a.mask = v.a[GLIDE_MASK]; a.bed = v.a[GLIDE_BED]; a.B = v.a[GLIDE_B];
        a.beta = v.a[GLIDE_BETA];
        a.ru = v.a[L.r[0]]; a.rv = v.a[L.r[1]]; a.rH = v.a[L.r[2]];
        a.xu = v.a[L.x[0]]; a.xv = v.a[L.x[1]]; a.xH = v.a[L.x[2]];
        a.f = blk[l];
        a.plane = size_t(v.ny) * v.pc;
        a.pitch = v.pc;
        a.err = err_dev;
        a.p = physr(l, dt, false);
        a.omega = R(c.omega); a.ssa_damping = R(c.ssa_damping); a.mc_damping = R(c.mc_damping);
        a.ny = v.ny; a.nx = v.nx;
        return a;
    }

    void block_factor(int l, double dt, const Lin& L, cudaStream_t s) {
        BlockArgs<R> a = block_args(l, dt, L);
        dim3 g(lv[l].blocks_x(), lv[l].blocks_y());
        const double bytes = lb(l, 9) + factor_bytes(l, L.tr);  // state read, 25 factor planes written
        if (record(G_BLOCK_FACTOR, L.tr ? 1 : 0, g, a, bytes)) {
            attach_maps(box_maps(l, kStateBoxes));
            return;
        }
        const BoxMaps<7> m = box_maps(l, kStateBoxes);
        if (L.tr) k_block_factor<R, true><<<g, kTile * kTile, 0, s>>>(a, m);
        else k_block_factor<R, false><<<g, kTile * kTile, 0, s>>>(a, m);
        counted("block_factor", bytes);
    }

    // n linear smoother sweeps (residual, then block solve and update); the
    // factors are refreshed first unless the caller just did
    void lin_sweeps(int l, double dt, int n, const Lin& L, cudaStream_t s, bool factor = true) {
        if (n <= 0) return;
        if (factor) block_factor(l, dt, L, s);
        BlockArgs<R> a = block_args(l, dt, L);
        dim3 g(lv[l].blocks_x(), lv[l].blocks_y());
        for (int k = 0; k < n; ++k) {
            lin_residual(l, dt, L, false, s);
            block_sweep(l, a, L.tr, g, s);
        }
    }

    // the 25 factor planes of level l
    double factor_bytes(int l, bool tr) const {
        const double per_cell = tr ? FactorStore<R, true>::kPlanes * sizeof(typename FactorStore<R, true>::type)
                                   : FactorStore<R, false>::kPlanes * sizeof(typename FactorStore<R, false>::type);
        return lb(l, per_cell / double(sizeof(R)));
    }

    // 25 factors, r, x read; x written
    void block_sweep(int l, const BlockArgs<R>& a, bool tr, dim3 g, cudaStream_t s) {
        const double bytes = lb(l, 9) + factor_bytes(l, tr);
        if (record(G_BLOCK_SWEEP, tr ? 1 : 0, g, a, bytes)) return;
        if (tr) k_block_sweep<R, true><<<g, kSweepThreads, 0, s>>>(a);
        else k_block_sweep<R, false><<<g, kSweepThreads, 0, s>>>(a);
        counted("linear_sweep", bytes);
    }

    void adj_sweeps(int l, double dt, int n, cudaStream_t s) { lin_sweeps(l, dt, n, adj_sys(), s); }

    // one launch of the linear smoother's block factorisation (part 0) or of
    // its block sweep on the current residual (part 1), nothing else
    void block_part(int l, double dt, bool adjoint, int part, cudaStream_t s) {
        ensure_blocks();
        const Lin L = adjoint ? adj_sys() : tan_sys();
        if (part == 0) {
            block_factor(l, dt, L, s);
            return;
        }
        BlockArgs<R> a = block_args(l, dt, L);
        block_sweep(l, a, L.tr, dim3(lv[l].blocks_x(), lv[l].blocks_y()), s);
    }

    // glide/multigrid.py:905-973 (linear FAS)
    void lin_vcycle(int l, bool finest, double dt, const Lin& L, cudaStream_t s) {
        const glide_fas_config& c = fas[L.cfg];
        block_factor(l, dt, L, s);  // the state is fixed for this visit of level l
        if (l == n_levels - 1) {
            lin_sweeps(l, dt, c.coarsest_steps, L, s, false);
            return;
        }
        Level<R>& n = lv[l + 1];
        lin_sweeps(l, dt, c.pre_steps, L, s, false);
        // the residual reads level l only: state, unknowns and residual are
        // restricted together after it, in one launch
        lin_residual(l, dt, L, false, s);
        {
            const RJob jobs[12] = {{GLIDE_U, -1, -1}, {GLIDE_V, -1, -1}, {GLIDE_H, -1, -1},
                                   {GLIDE_H_PREV, -1, -1}, {GLIDE_PHI, -1, -1}, {GLIDE_MASK, -1, -1},
                                   {L.x[0], L.w[0], -1}, {L.x[1], L.w[1], -1}, {L.x[2], L.w[2], -1},
                                   {L.r[0], -1, -1}, {L.r[1], -1, -1}, {L.r[2], -1, -1}};
            restrict_batch(l, jobs, 12, s);
        }
        // coarse right-hand side f_c = Op_c(x_c) - R r, in one pass
        lin_op(l + 1, dt, L, L.f, L.r, false, false, false, s);
        lin_vcycle(l + 1, false, dt, L, s);
        correct3(l, {L.x[0], L.x[1], L.x[2]}, {L.w[0], L.w[1], L.w[2]}, {kFaceU, kFaceV, kCellMax}, 1, s);
        lin_sweeps(l, dt, c.post_steps, L, s, false);
        if (finest) lin_sweeps(l, dt, c.finest_steps, L, s, false);
    }

    void adj_vcycle(int l, bool finest, double dt, cudaStream_t s) { lin_vcycle(l, finest, dt, adj_sys(), s); }

    // ----------------------------------------------------- Newton cycle
    // One outer step of Newton's method on the binary64 residual.  On entry
    // R_* hold the unmasked residual of the current state and MASK its active
    // set (the smoother's rule H - dt r_H <= gamma; see newton_prologue).  The
    // tangent system J(x) e = -r (identity rows on active cells and Dirichlet
    // faces) is solved by `tangent_vcycles` V-cycles of the linear multigrid --
    // on the binary32 shadow for a mixed handle, on this hierarchy otherwise --
    // then x <- x + e with H floored at gamma, and one binary64 residual pass
    // recomputes phi, the residual, the next active set and the masked norms.
    int tangent_vcycles = 1;

    void newton_prologue(int l, double dt, bool norms, cudaStream_t s) {
        residual(l, dt, true, false, false, false, GLIDE_R_U, GLIDE_R_V, GLIDE_R_H, nullptr, norms, s, true);
    }

    template <class T>
    void newton_cycle_on(Solver<T>& ts, int l, double dt, cudaStream_t s) {
        Level<R>& D = lv[l];
        Level<T>& F = ts.lv[l];
        if constexpr (!std::is_same<T, R>::value) {
            not_recordable("a mixed-precision Newton step");
            push_to_shadow(l, {GLIDE_U, GLIDE_V, GLIDE_H, GLIDE_PHI, GLIDE_MASK}, false, s);
        }
        const TangentRhsArgs<T, R> ta{F.a[F_TF_U], F.a[F_TF_V], F.a[F_TF_H], D.a[GLIDE_R_U], D.a[GLIDE_R_V],
                                      D.a[GLIDE_R_H], D.a[GLIDE_H], D.a[GLIDE_GAMMA], D.a[GLIDE_MASK], D.ny, D.nx};
        const double ta_bytes = double(D.ny) * D.nx * (6 * sizeof(R) + 3 * sizeof(T));
        if (!record(G_TANGENT_RHS, 0, pw_grid(D.ny + 1, D.nx + 1), ta, ta_bytes)) {
            k_tangent_rhs<T, R><<<pw_grid(D.ny + 1, D.nx + 1), 256, 0, s>>>(ta);
            counted("tangent_rhs", ta_bytes);
        }
        for (int fld : {F_E_U, F_E_V, F_E_H}) ts.fill(F.a[fld], T(0), s);
        for (int k = 0; k < tangent_vcycles; ++k) ts.lin_vcycle(l, true, dt, Solver<T>::tan_sys(), s);
        const NewtonUpdateArgs<R, T> na{D.a[GLIDE_U], D.a[GLIDE_V], D.a[GLIDE_H], D.a[GLIDE_GAMMA],
                                        F.a[F_E_U], F.a[F_E_V], F.a[F_E_H], D.ny, D.nx};
        const double na_bytes = double(D.ny) * D.nx * (7 * sizeof(R) + 3 * sizeof(T));
        if (!record(G_NEWTON_UPDATE, 0, pw_grid(D.ny + 1, D.nx + 1), na, na_bytes)) {
            k_newton_update<R, T><<<pw_grid(D.ny + 1, D.nx + 1), 256, 0, s>>>(na);
            counted("newton_update", na_bytes);
        }
        residual(l, dt, true, false, false, false, GLIDE_R_U, GLIDE_R_V, GLIDE_R_H, nullptr, true, s, true);
    }

    void newton_cycle(int l, double dt, cudaStream_t s) {
        if constexpr (sizeof(R) == 8) {
            if (lo) {
                newton_cycle_on(*lo, l, dt, s);
                return;
            }
        }
        newton_cycle_on(*this, l, dt, s);
    }

    void backward(double dt, int start, int grad_mask, glide_stats* st, cudaStream_t s) {
        check_level(start);
        check_quirks();
        ensure_blocks();
        if constexpr (sizeof(R) == 8) {
            if (lo) lo->ensure_blocks();
        }
        if constexpr (sizeof(R) == 8) {
            if (lo) {
                backward_mixed(dt, start, grad_mask, st, s);
                return;
            }
        }
        adj_residual(start, dt, true, s);
        double nr[4];
        read_norms(nr, s);
        solve_loop(1, start, dt, nr, st, s);
        gradients(start, dt, grad_mask, s);
    }

    void gradients(int l, double dt, int mask, cudaStream_t s) {
        Level<R>& v = lv[l];
        GradArgs<R> a;
        a.u = v.a[GLIDE_U]; a.v = v.a[GLIDE_V]; a.H = v.a[GLIDE_H];
        a.phi = v.a[GLIDE_PHI]; a.bed = v.a[GLIDE_BED]; a.beta = v.a[GLIDE_BETA];
        a.lu = v.a[GLIDE_LAMBDA_U]; a.lv = v.a[GLIDE_LAMBDA_V]; a.lH = v.a[GLIDE_LAMBDA_H];
        a.g_beta = (mask & GLIDE_GRAD_BETA_BIT) ? v.a[GLIDE_GRAD_BETA] : Arr<R>();
        a.g_bed = (mask & GLIDE_GRAD_BED_BIT) ? v.a[GLIDE_GRAD_BED] : Arr<R>();
        a.g_Hp = (mask & GLIDE_GRAD_H_PREV_BIT) ? v.a[GLIDE_GRAD_H_PREV] : Arr<R>();
        a.g_smb = (mask & GLIDE_GRAD_SMB_BIT) ? v.a[GLIDE_GRAD_SMB] : Arr<R>();
        a.p = physr(l, dt, false);
        a.dt = R(dt);
        a.ny = v.ny; a.nx = v.nx;
        const double bytes = lb(l, 9 + __builtin_popcount(unsigned(mask) & 15u));
        if (record(G_GRADIENTS, 0, pw_grid(v.ny, v.nx), a, bytes)) return;
        k_gradients<R><<<pw_grid(v.ny, v.nx), 256, 0, s>>>(a);
        counted("gradients", bytes);
    }
};

// ================================================================== groups
// One solver cycle run over several hierarchies of one value type in grouped
// launches (group.cuh).  A plan is every member's cycle as its own Solver
// code issues it, recorded instead of launched, then merged: the member with
// the most launches left sets the next kind, and every member whose next
// launch is of that kind joins it.  Each member's launches keep their order,
// so a member computes exactly what its own solve computes.  A plan is
// captured once as a CUDA graph and replayed; the graph of a cycle ends in
// the device-side convergence test.
struct GroupBase {
    virtual ~GroupBase() {}
    virtual void invalidate() = 0;  // rebuild every plan on the next call
    int dtype = GLIDE_F64;
    int waves = 0;  // grid of a grouped launch: waves x resident blocks (0: one block per tile)
    int spoil_maps = 0;  // GLIDE_GROUP_TUNE_SPOIL_MAPS: upload the staging maps without their tag
    long long launches = 0;  // grouped launches issued (graph replays included)
    int shape[4] = {0, 0, 0, 0};  // last forward / adjoint cycle: grouped launches, member launches
    virtual void forward(double dt, int start, glide_stats* st, cudaStream_t s) = 0;
    virtual void backward(double dt, int start, int grad_mask, glide_stats* st, cudaStream_t s) = 0;
};

template <class R>
struct GroupRun : GroupBase {
    std::vector<Solver<R>*> members;
    GroupMember* dev = nullptr;   // device solve state, one per member
    int* flags = nullptr;         // device run flags; flags[n], flags[n + 1]: running members, their sections
    int* running_host = nullptr;  // pinned copy of those two words
    std::vector<GroupMember> host;
    cudaStream_t own_stream = nullptr;

    struct Launch {
        int op, variant, when;
        std::vector<std::pair<int, const RecOp*>> items;  // (member, its recorded launch)
        const unsigned char* dev_maps = nullptr;           // the items' staging maps on the device
    };
    // A plan is a list of sections: grouped launches predicated on a flag bit,
    // or one phase of the device-side decisions.
    struct Section {
        int control;  // a GroupPhase, or -1
        int when;     // flag bits of the members whose launches run (0: every member)
        std::function<void(Solver<R>&, int)> body;  // records member k's launches
        int tag = -1;  // byte accounting: one of the T_* kinds below
    };
    // forward cycle sections whose algorithmic bytes are accounted per use
    enum { T_PRO, T_BACKUP, T_FAS, T_NEWTON, T_UNDO, T_COUNT };
    std::vector<double> sec_bytes[T_COUNT];  // per member, one pass
    struct Plan {
        std::vector<int> control;                      // per section
        std::vector<std::vector<std::vector<RecOp>>> rec;  // [section][member]
        std::vector<std::vector<Launch>> launches;     // [section]
        std::vector<std::vector<double>> bytes;        // [section][member]: algorithmic bytes
        cudaGraphExec_t exec = nullptr;
        long long nodes = 0;
        std::vector<void*> buffers;  // the launches' staging maps on the device
        std::vector<unsigned> versions;
        double dt = 0;
        int start = -1, extra = 0;
        bool valid = false;
    };
    enum { P_FWD_PRO, P_ADJ_PRO, P_ADJ_CYCLE, P_GRAD, P_COUNT };
    Plan plans[P_COUNT];
    // forward cycles by the sections they hold (bits: FASCD, Newton, prologue):
    // each cycle replays the variant holding just what the running members need
    Plan fwd_cycles[8];

    explicit GroupRun(std::vector<Solver<R>*> m) : members(std::move(m)) {
        dtype = sizeof(R) == 8 ? GLIDE_F64 : GLIDE_F32;
        const int n = int(members.size());
        host.resize(n);
        GCU(cudaMalloc(&dev, sizeof(GroupMember) * n));
        GCU(cudaMalloc(&flags, sizeof(int) * (n + 2)));
        GCU(cudaMemset(flags, 0, sizeof(int) * (n + 2)));
        GCU(cudaMallocHost(&running_host, 2 * sizeof(int)));
        for (auto& b : sec_bytes) b.assign(n, 0.0);
        GCU(cudaDeviceSynchronize());
    }

    ~GroupRun() override {
        for (Plan& p : plans) {
            if (p.exec) cudaGraphExecDestroy(p.exec);
            for (void* b : p.buffers) cudaFree(b);
        }
        for (Plan& p : fwd_cycles) {
            if (p.exec) cudaGraphExecDestroy(p.exec);
            for (void* b : p.buffers) cudaFree(b);
        }
        if (own_stream) cudaStreamDestroy(own_stream);
        if (running_host) cudaFreeHost(running_host);
        if (flags) cudaFree(flags);
        if (dev) cudaFree(dev);
    }

    void invalidate() override {
        for (Plan& p : plans) p.valid = false;
        for (Plan& p : fwd_cycles) p.valid = false;
    }

    // the plan's device copies of staging maps (its graph is gone or idle)
    void release(Plan& P) {
        for (void* b : P.buffers) cudaFree(b);
        P.buffers.clear();
    }

    // Bytes of the staging maps an op kind records (0: none).
    static size_t maps_bytes(int op) {
        switch (op) {
            case G_RESIDUAL: return sizeof(BoxMaps<OpMaps<GResidual<R>>::n>);
            case G_VJP: return sizeof(BoxMaps<OpMaps<GVjp<R>>::n>);
            case G_JVP: return sizeof(BoxMaps<OpMaps<GJvp<R>>::n>);
            case G_BLOCK_FACTOR: return sizeof(BoxMaps<OpMaps<GBlockFactor<R, false>>::n>);
            default: return 0;
        }
    }

    // Clear the tag of the staging maps at p (op's kind of maps).
    template <int N>
    static void untag(unsigned char* p) {
        BoxMaps<N> m;
        std::memcpy(static_cast<void*>(&m), p, sizeof(m));
        m.tag = 0;
        std::memcpy(p, static_cast<const void*>(&m), sizeof(m));
    }
    static void untag(int op, unsigned char* p) {
        switch (op) {
            case G_RESIDUAL: return untag<OpMaps<GResidual<R>>::n>(p);
            case G_VJP: return untag<OpMaps<GVjp<R>>::n>(p);
            case G_JVP: return untag<OpMaps<GJvp<R>>::n>(p);
            case G_BLOCK_FACTOR: return untag<OpMaps<GBlockFactor<R, false>>::n>(p);
            default: return;
        }
    }

    // Copy each stencil launch's staging maps into one device array (before
    // a capture: no allocation may happen inside it).  The copies run on the
    // stream the plan's graph will run on, and the call waits for them: a
    // copy on the legacy stream would not be ordered before the kernels on a
    // non-blocking stream, which could then read the array before it holds
    // the maps.
    void upload_maps(Plan& P, cudaStream_t s) {
        for (auto& sec : P.launches)
            for (Launch& L : sec) {
                const size_t b = maps_bytes(L.op);
                if (!b || L.dev_maps) continue;
                std::vector<unsigned char> host(b * L.items.size());
                for (size_t q = 0; q < L.items.size(); ++q) {
                    const RecOp& r = *L.items[q].second;
                    if (r.maps.size() != b) fail(GLIDE_ERR_STATE, "a stencil launch was recorded without its maps");
                    std::memcpy(host.data() + q * b, r.maps.data(), b);
                    if (spoil_maps) untag(L.op, host.data() + q * b);
                }
                void* d = nullptr;
                GCU(cudaMalloc(&d, host.size()));
                P.buffers.push_back(d);
                GCU(cudaMemcpyAsync(d, host.data(), host.size(), cudaMemcpyHostToDevice, s));
                GCU(cudaStreamSynchronize(s));
                L.dev_maps = static_cast<const unsigned char*>(d);
            }
    }

    // Record every member's sections into P (unless P is current) and merge
    // each section's launches across members: the member with the most
    // launches left sets the next kind, every member whose next launch is of
    // that kind joins it.
    void build(Plan& P, double dt, int start, int extra, const std::vector<Section>& secs) {
        std::vector<unsigned> v;
        for (auto* m : members) v.push_back(m->version);
        if (P.valid && P.dt == dt && P.start == start && P.extra == extra && P.versions == v) return;
        if (P.exec) {
            cudaGraphExecDestroy(P.exec);
            P.exec = nullptr;
        }
        release(P);
        P.valid = false;
        const int n = int(members.size());
        const size_t ns = secs.size();
        P.control.assign(ns, -1);
        P.rec.assign(ns, std::vector<std::vector<RecOp>>(n));
        P.launches.assign(ns, {});
        P.bytes.assign(ns, std::vector<double>(n, 0.0));
        for (size_t q = 0; q < ns; ++q) {
            P.control[q] = secs[q].control;
            if (secs[q].control >= 0) continue;
            for (int k = 0; k < n; ++k) {
                Solver<R>& m = *members[k];
                m.rec = &P.rec[q][k];
                try {
                    secs[q].body(m, k);
                } catch (...) {
                    m.rec = nullptr;
                    throw;
                }
                m.rec = nullptr;
                for (const RecOp& r : P.rec[q][k]) P.bytes[q][k] += r.bytes;
                if (secs[q].tag >= 0) sec_bytes[secs[q].tag][k] = P.bytes[q][k];
            }
            std::vector<size_t> pos(n, 0);
            for (;;) {
                int pick = -1;
                size_t most = 0;
                for (int k = 0; k < n; ++k)
                    if (P.rec[q][k].size() - pos[k] > most) {
                        most = P.rec[q][k].size() - pos[k];
                        pick = k;
                    }
                if (pick < 0) break;
                const RecOp& h = P.rec[q][pick][pos[pick]];
                Launch L{h.op, h.variant, secs[q].when, {}};
                for (int k = 0; k < n; ++k) {
                    if (pos[k] == P.rec[q][k].size()) continue;
                    const RecOp& r = P.rec[q][k][pos[k]];
                    if (r.op == h.op && r.variant == h.variant) {
                        L.items.push_back({k, &r});
                        ++pos[k];
                    }
                }
                P.launches[q].push_back(std::move(L));
            }
        }
        P.versions = v;
        P.dt = dt;
        P.start = start;
        P.extra = extra;
        P.valid = true;
    }

    // One launch per N items of L (N: what fits the parameter space): one
    // block per tile of every item (waves == 0), or `waves` waves of resident
    // blocks striding over the tiles; blocks of an item whose member does not
    // run this cycle return at once.
    template <class Op>
    long long issue_op(const Launch& L, cudaStream_t s) {
        using A = typename Op::Args;
        constexpr int N = group_capacity<A>();
        static_assert(sizeof(GroupParams<A, N>) <= 32764, "kernel parameters over the limit");
        static const long long wave = [] {
            int dev = 0, sms = 0, per_sm = 0;
            GCU(cudaGetDevice(&dev));
            GCU(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
            GCU(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_group_waves<Op, N>, Op::kThreads, 0));
            return (long long)sms * std::max(per_sm, 1);
        }();
        long long issued = 0;
        for (size_t base = 0; base < L.items.size(); base += N) {
            auto P = std::make_unique<GroupParams<A, N>>();
            P->flags = flags;
            P->when = L.when;
            constexpr size_t mb = OpMaps<Op>::n ? sizeof(BoxMaps<OpMaps<Op>::n ? OpMaps<Op>::n : 1>) : 0;
            if (mb && !L.dev_maps) fail(GLIDE_ERR_STATE, "staging maps not on the device");
            P->maps = mb ? L.dev_maps + base * mb : nullptr;
            P->maps_stride = unsigned(mb);
            long long nb = 0;
            int k = 0;
            for (size_t q = base; q < L.items.size() && k < N; ++q, ++k) {
                const RecOp& r = *L.items[q].second;
                if (r.args.size() != sizeof(A)) fail(GLIDE_ERR_STATE, "recorded arguments of the wrong size");
                const long long blocks = (long long)r.gx * r.gy * r.gz;
                if (blocks > 0x7fffffffLL) fail(GLIDE_ERR_SHAPE, "grouped launch over 2^31 tiles");
                P->item[k] = GroupItem{int(nb), r.gx, r.gy, L.items[q].first};
                std::memcpy(static_cast<void*>(&P->args[k]), r.args.data(), sizeof(A));
                nb += blocks;
            }
            if (nb > 0x7fffffffLL) fail(GLIDE_ERR_SHAPE, "grouped launch over 2^31 tiles");
            if (nb == 0) continue;  // no tiles (a block per tile would run one of an empty item)
            P->n = k;
            if (waves > 0) {
                const long long grid = std::min(nb, waves * wave);
                k_group_waves<Op, N><<<unsigned(std::max(grid, 1LL)), Op::kThreads, 0, s>>>(*P, int(nb));
            } else {
                k_group<Op, N><<<unsigned(std::max(nb, 1LL)), Op::kThreads, 0, s>>>(*P);
            }
            check_launch("grouped launch");
            ++issued;
        }
        return issued;
    }

    long long issue(const Launch& L, cudaStream_t s) {
        const int v = L.variant;
        switch (L.op) {
            case G_SNAPSHOT: return issue_op<GSnapshot<R>>(L, s);
            case G_RESTRICT: return issue_op<GRestrict<R>>(L, s);
            case G_RESTRICT_BATCH: return issue_op<GRestrictBatch<R>>(L, s);
            case G_CORRECT_BATCH: return issue_op<GCorrectBatch<R>>(L, s);
            case G_GROUNDED: return issue_op<GGrounded<R>>(L, s);
            case G_COPY: return issue_op<GCopy<R>>(L, s);
            case G_FILL: return issue_op<GFill<R>>(L, s);
            case G_SET_RHS: return issue_op<GSetRhs<R>>(L, s);
            case G_TANGENT_RHS: return issue_op<GTangentRhs<R>>(L, s);
            case G_NEWTON_UPDATE: return issue_op<GNewtonUpdate<R>>(L, s);
            case G_GRADIENTS: return issue_op<GGradients<R>>(L, s);
            case G_NORMS: return issue_op<GNorms>(L, s);
            case G_RESIDUAL: return issue_op<GResidual<R>>(L, s);
            case G_VJP: return issue_op<GVjp<R>>(L, s);
            case G_JVP: return issue_op<GJvp<R>>(L, s);
            case G_SWEEP:
                if (v & 2) return (v & 1) ? issue_op<GSweep<R, true, 2>>(L, s) : issue_op<GSweep<R, false, 2>>(L, s);
                return (v & 1) ? issue_op<GSweep<R, true, 1>>(L, s) : issue_op<GSweep<R, false, 1>>(L, s);
            case G_BLOCK_FACTOR:
                return v ? issue_op<GBlockFactor<R, true>>(L, s) : issue_op<GBlockFactor<R, false>>(L, s);
            case G_BLOCK_SWEEP:
                return v ? issue_op<GBlockSweep<R, true>>(L, s) : issue_op<GBlockSweep<R, false>>(L, s);
            default: fail(GLIDE_ERR_STATE, "unknown grouped launch kind");
        }
        return 0;
    }

    // replay P's graph, capturing it first
    void run_plan(Plan& P, cudaStream_t s) {
        const int n = int(members.size());
        if (!P.exec) {
            std::lock_guard<std::mutex> lock(g_capture_mu);
            upload_maps(P, s);
            cudaGraph_t g = nullptr;
            long long nodes = 0;
            GCU(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
            try {
                for (size_t q = 0; q < P.control.size(); ++q) {
                    if (P.control[q] >= 0) {
                        k_group_control<<<1, kGroupControlThreads, 0, s>>>(dev, flags, n, P.control[q],
                                                                            flags + n);
                        check_launch("group_control");
                        ++nodes;
                    } else {
                        for (const Launch& L : P.launches[q]) nodes += issue(L, s);
                    }
                }
            } catch (...) {
                cudaStreamEndCapture(s, &g);
                if (g) cudaGraphDestroy(g);
                throw;
            }
            GCU(cudaStreamEndCapture(s, &g));
            const cudaError_t e = cudaGraphInstantiate(&P.exec, g, 0);
            cudaGraphDestroy(g);
            if (e != cudaSuccess) fail(GLIDE_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(e));
            P.nodes = nodes;
        }
        GCU(cudaGraphLaunch(P.exec, s));
        launches += P.nodes;
    }

    cudaStream_t stream_for(cudaStream_t s) {
        // the legacy default stream cannot be captured (see Solver::cycle_and_check)
        if (s) return s;
        if (!own_stream) GCU(cudaStreamCreate(&own_stream));
        return own_stream;
    }

    void check_members(int start) {
        for (auto* m : members) {
            m->check_level(start);
            m->check_quirks();
            if constexpr (sizeof(R) == 8) {
                if (m->lo) fail(GLIDE_ERR_STATE, "mixed-precision hierarchies have no grouped form");
            }
        }
    }

    static Section launches_of(int when, std::function<void(Solver<R>&, int)> body, int tag = -1) {
        return Section{-1, when, std::move(body), tag};
    }
    static Section control(int phase) { return Section{phase, 0, nullptr}; }

    // the prologue plan, then cycles -- cycle(sections) picks the plan for the
    // section bits the running members need -- until no member runs; the
    // members' final device state is left in `host`
    void solve(Plan& pro, const std::function<Plan&(int)>& cycle, int cfg, bool forward, cudaStream_t s) {
        const int n = int(members.size());
        int max_cycles = 0;
        for (int k = 0; k < n; ++k) {
            Solver<R>& m = *members[k];
            const glide_fas_config& c = m.fas[cfg];
            GroupMember& g = host[k];
            std::memset(static_cast<void*>(&g), 0, sizeof(g));
            g.norms = m.norms_dev;
            g.err = m.err_dev;
            g.rtol = c.relative_tolerance;
            g.atol = c.absolute_tolerance;
            g.max_cycles = c.maximum_vcycles;
            g.newton = forward && m.forward_method == 1;
            g.newton_switch = m.newton_switch;
            g.stall_ratio = m.newton_stall_ratio;
            max_cycles = std::max(max_cycles, c.maximum_vcycles);
        }
        GCU(cudaMemcpyAsync(dev, host.data(), sizeof(GroupMember) * n, cudaMemcpyHostToDevice, s));
        run_plan(pro, s);  // ends with the GC_INIT phase
        for (int it = 0;; ++it) {
            GCU(cudaMemcpyAsync(running_host, flags + n, 2 * sizeof(int), cudaMemcpyDeviceToHost, s));
            GCU(cudaStreamSynchronize(s));
            if (running_host[0] == 0 || it >= max_cycles) break;
            run_plan(cycle(running_host[1]), s);  // ends with the GC_END phase
        }
        GCU(cudaMemcpyAsync(host.data(), dev, sizeof(GroupMember) * n, cudaMemcpyDeviceToHost, s));
        GCU(cudaStreamSynchronize(s));
    }

    // statistics and the members' own records of the solve
    void finish(const Plan& pro, int cfg, glide_stats* st, const std::function<double(int)>& bytes,
                cudaStream_t s) {
        int bad = -1, late = -1, word = 0;
        for (size_t k = 0; k < members.size(); ++k) {
            const GroupMember& g = host[k];
            Solver<R>& m = *members[k];
            if (g.status == GS_STAGING) {
                // clear the word, so the member's next solve starts clean
                GCU(cudaMemsetAsync(m.err_dev, 0, sizeof(int), s));
                GCU(cudaStreamSynchronize(s));
                if (late < 0) {
                    late = int(k);
                    word = g.err_word;
                }
            }
            if (st) {
                glide_stats& o = st[k];
                std::memset(&o, 0, sizeof(o));
                o.vcycles = g.cycles;
                o.initial_norm = g.r0;
                o.final_norm = g.last;
                for (int q = 0; q < 3; ++q) o.norms[q] = g.last_norms[q];
                for (int q = 0; q <= g.cycles && q < GLIDE_MAX_HISTORY; ++q) o.history[q] = g.history[q];
            }
            double b = bytes(int(k));
            for (const auto& sec : pro.bytes) b += sec[k];
            m.traffic(b);
            m.newton_rejects += g.rejects;
            const double rel = g.r0 > 0 ? g.last / g.r0 : 0.0;
            const glide_fas_config& c = m.fas[cfg];
            m.last_not_converged = !(rel <= c.relative_tolerance || g.last <= c.absolute_tolerance);
            m.last_relative = rel;
            m.last_cycles = g.cycles;
            if (g.status == GS_NONFINITE && bad < 0) bad = int(k);
        }
        if (late >= 0 && (word & kStageBadMaps))
            fail(GLIDE_ERR_STATE, "member " + std::to_string(late) + ": staging maps failed their check");
        if (late >= 0)
            fail(GLIDE_ERR_TIMEOUT, "member " + std::to_string(late) + ": a bounded wait for staged tiles gave up");
        if (bad >= 0) fail(GLIDE_ERR_NONFINITE, "member " + std::to_string(bad) + ": residual norm is not finite");
    }

    void note_shape(const Plan& P, int slot) {
        int grouped = 0;
        long long total = 0;
        for (size_t q = 0; q < P.control.size(); ++q) {
            grouped += int(P.launches[q].size());
            for (const auto& r : P.rec[q]) total += (long long)r.size();
        }
        shape[slot] = grouped;
        shape[slot + 1] = int(total);
    }

    void forward(double dt, int start, glide_stats* st, cudaStream_t s) override {
        s = stream_for(s);
        check_members(start);
        for (auto* m : members)
            if (m->forward_method == 1) m->ensure_blocks();
        auto is_newton = [&](int k) { return members[k]->forward_method == 1; };
        build(plans[P_FWD_PRO], dt, start, 0,
              {launches_of(0, [&](Solver<R>& m, int) {
                   m.set_rhs(start, dt, s);
                   m.residual(start, dt, true, true, false, false, GLIDE_R_U, GLIDE_R_V, GLIDE_R_H, nullptr, true,
                              s);
               }),
               control(GC_INIT)});
        auto save = [&](Solver<R>& m, int k, bool undo) {
            if (!is_newton(k)) return;
            Level<R>& L0 = m.lv[start];
            const int x[4] = {GLIDE_U, GLIDE_V, GLIDE_H, GLIDE_MASK}, b[4] = {F_BK_U, F_BK_V, F_BK_H, F_BK_MASK};
            for (int q = 0; q < 4; ++q) {
                if (undo) m.copy(L0.a[x[q]], L0.a[b[q]], s);
                else m.copy(L0.a[b[q]], L0.a[x[q]], s);
            }
        };
        // The per-hierarchy solve loop's sequence: the Newton prologue, the
        // state saved, a FASCD cycle or a Newton step, the step undone if its
        // residual grew, the convergence test and the next cycle's decision.
        int used[8] = {0};
        auto cycle = [&](int bits) -> Plan& {
            const int fas = bits & kGroupFas, newton = bits & kGroupNewton, pro = bits & kGroupPro;
            const int v = (fas ? 1 : 0) | (newton ? 2 : 0) | (pro ? 4 : 0);
            std::vector<Section> secs;
            if (pro) {
                secs.push_back(launches_of(kGroupPro, [&](Solver<R>& m, int k) {
                    if (is_newton(k)) m.newton_prologue(start, dt, true, s);
                }, T_PRO));
                secs.push_back(control(GC_MID));
            }
            if (newton) secs.push_back(launches_of(kGroupNewton, [&](Solver<R>& m, int k) { save(m, k, false); }, T_BACKUP));
            if (fas)
                secs.push_back(launches_of(kGroupFas, [&](Solver<R>& m, int) {
                    m.vcycle(start, true, dt, s);
                    m.residual(start, dt, true, true, false, true, GLIDE_R_U, GLIDE_R_V, GLIDE_R_H, nullptr, true, s);
                }, T_FAS));
            if (newton) {
                secs.push_back(launches_of(kGroupNewton, [&](Solver<R>& m, int k) {
                    if (is_newton(k)) m.newton_cycle(start, dt, s);
                }, T_NEWTON));
                secs.push_back(control(GC_POST));
                secs.push_back(launches_of(kGroupUndo, [&](Solver<R>& m, int k) { save(m, k, true); }, T_UNDO));
            }
            secs.push_back(control(GC_END));
            build(fwd_cycles[v], dt, start, 0, secs);
            ++used[v];
            return fwd_cycles[v];
        };
        solve(plans[P_FWD_PRO], cycle, 0, true, s);
        int most = 0;
        for (int v = 1; v < 8; ++v)
            if (used[v] > used[most]) most = v;
        if (used[most]) note_shape(fwd_cycles[most], 0);
        finish(plans[P_FWD_PRO], 0, st, [&](int k) {
            // FASCD cycles, Newton steps (state saved), prologues and undone steps
            const GroupMember& g = host[k];
            const int steps = g.cycles - g.fas_cycles;
            return g.fas_cycles * sec_bytes[T_FAS][k] + steps * (sec_bytes[T_BACKUP][k] + sec_bytes[T_NEWTON][k]) +
                   g.prologues * sec_bytes[T_PRO][k] + g.rejects * sec_bytes[T_UNDO][k];
        }, s);
    }

    void backward(double dt, int start, int grad_mask, glide_stats* st, cudaStream_t s) override {
        s = stream_for(s);
        check_members(start);
        for (auto* m : members) m->ensure_blocks();
        build(plans[P_ADJ_PRO], dt, start, 0,
              {launches_of(0, [&](Solver<R>& m, int) { m.adj_residual(start, dt, true, s); }), control(GC_INIT)});
        Plan& C = plans[P_ADJ_CYCLE];
        build(C, dt, start, 0,
              {launches_of(kGroupRun,
                           [&](Solver<R>& m, int) {
                               m.adj_vcycle(start, true, dt, s);
                               m.adj_residual(start, dt, true, s);
                           }),
               control(GC_END)});
        build(plans[P_GRAD], dt, start, grad_mask,
              {launches_of(0, [&](Solver<R>& m, int) { m.gradients(start, dt, grad_mask, s); })});
        note_shape(C, 2);
        solve(plans[P_ADJ_PRO], [&](int) -> Plan& { return C; }, 1, false, s);
        run_plan(plans[P_GRAD], s);
        finish(plans[P_ADJ_PRO], 1, st, [&](int k) { return host[k].cycles * C.bytes[0][k] + plans[P_GRAD].bytes[0][k]; },
               s);
    }
};

}  // namespace glide

// ====================================================================== C ABI
using namespace glide;

struct glide_solver {
    std::unique_ptr<SolverBase> impl;
};

struct glide_group_s {
    std::unique_ptr<GroupBase> impl;
};

namespace {

template <class F>
int guarded(F&& f) {
    try {
        f();
        return GLIDE_OK;
    } catch (const Fail& e) {
        return e.code;
    } catch (const std::exception& e) {
        g_err = e.what();
        return GLIDE_ERR_STATE;
    }
}

template <class F>
void dispatch(glide_handle h, F&& f) {
    if (!h || !h->impl) fail(GLIDE_ERR_ARG, "null handle");
    if (h->impl->dtype == GLIDE_F64) f(*static_cast<Solver<double>*>(h->impl.get()));
    else f(*static_cast<Solver<float>*>(h->impl.get()));
}

cudaStream_t S(void* p) { return static_cast<cudaStream_t>(p); }

template <class R>
Arr<R>& field_arr(Solver<R>& s, int field, int level) {
    s.check_level(level);
    if (field < 0 || field >= GLIDE_N_PUBLIC_FIELDS) fail(GLIDE_ERR_ARG, "unknown field id");
    return s.lv[level].a[field];
}

}  // namespace

extern "C" {

const char* glide_last_error(void) { return g_err.c_str(); }
int glide_version(void) { return 1; }

int glide_create(int ny, int nx, double dx, int n_levels, int dtype, glide_handle* out) {
    return guarded([&] {
        if (!out) fail(GLIDE_ERR_ARG, "out is null");
        *out = nullptr;
        if (ny <= 0 || nx <= 0 || n_levels <= 0 || !(dx > 0)) fail(GLIDE_ERR_ARG, "bad grid arguments");
        if (n_levels > 16) fail(GLIDE_ERR_ARG, "too many levels");
        const int d = 1 << (n_levels - 1);
        if (ny % d || nx % d)
            fail(GLIDE_ERR_SHAPE, "ny and nx must be divisible by 2^(n_levels-1)");
        if ((ny >> (n_levels - 1)) < 2 || (nx >> (n_levels - 1)) < 2)
            fail(GLIDE_ERR_SHAPE, "coarsest level must have at least 2x2 cells");
        auto h = std::make_unique<glide_solver>();
        if (dtype == GLIDE_F64) {
            h->impl = std::make_unique<Solver<double>>(ny, nx, dx, n_levels);
        } else if (dtype == GLIDE_F32) {
            h->impl = std::make_unique<Solver<float>>(ny, nx, dx, n_levels);
        } else if (dtype == GLIDE_MIXED) {
            auto d = std::make_unique<Solver<double>>(ny, nx, dx, n_levels);
            d->lo = std::make_unique<Solver<float>>(ny, nx, dx, n_levels);
            d->forward_method = 1;  // FAS in binary32 stalls at its rounding floor: finish with Newton
            h->impl = std::move(d);
        } else {
            fail(GLIDE_ERR_ARG, "dtype must be GLIDE_F64, GLIDE_F32 or GLIDE_MIXED");
        }
        *out = h.release();
    });
}

int glide_destroy(glide_handle h) {
    return guarded([&] { delete h; });
}

int glide_level_shape(glide_handle h, int level, int* ny, int* nx, double* dx) {
    return guarded([&] {
        dispatch(h, [&](auto& s) {
            s.check_level(level);
            if (ny) *ny = s.lv[level].ny;
            if (nx) *nx = s.lv[level].nx;
            if (dx) *dx = s.lv[level].dx;
        });
    });
}

int glide_field_ptr(glide_handle h, int field, int level, void** ptr, int* rows, int* cols, int* pitch) {
    return guarded([&] {
        dispatch(h, [&](auto& s) {
            auto& a = field_arr(s, field, level);
            if (ptr) *ptr = a.p;
            if (rows) *rows = a.rows;
            if (cols) *cols = a.cols;
            if (pitch) *pitch = a.pitch;
        });
    });
}

int glide_set_field(glide_handle h, int field, int level, const void* src, int src_ld, int src_on_host,
                    int restrict_down, void* stream) {
    return guarded([&] {
        if (!src) fail(GLIDE_ERR_ARG, "src is null");
        dispatch(h, [&](auto& s) {
            using R = std::remove_reference_t<decltype(*s.lv[0].a[0].p)>;
            auto& a = field_arr(s, field, level);
            const int ld = src_ld > 0 ? src_ld : a.cols;
            if (ld < a.cols) fail(GLIDE_ERR_ARG, "src_ld smaller than the field's columns");
            GCU(cudaMemcpy2DAsync(a.p, size_t(a.pitch) * sizeof(R), src, size_t(ld) * sizeof(R),
                                  size_t(a.cols) * sizeof(R), a.rows,
                                  src_on_host ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice, S(stream)));
            if (restrict_down)
                for (int l = level; l + 1 < s.n_levels; ++l) s.restrict_field(field, l, S(stream));
            if (src_on_host) GCU(cudaStreamSynchronize(S(stream)));
        });
    });
}

int glide_get_field(glide_handle h, int field, int level, void* dst, int dst_ld, int dst_on_host, void* stream) {
    return guarded([&] {
        if (!dst) fail(GLIDE_ERR_ARG, "dst is null");
        dispatch(h, [&](auto& s) {
            using R = std::remove_reference_t<decltype(*s.lv[0].a[0].p)>;
            auto& a = field_arr(s, field, level);
            const int ld = dst_ld > 0 ? dst_ld : a.cols;
            if (ld < a.cols) fail(GLIDE_ERR_ARG, "dst_ld smaller than the field's columns");
            GCU(cudaMemcpy2DAsync(dst, size_t(ld) * sizeof(R), a.p, size_t(a.pitch) * sizeof(R),
                                  size_t(a.cols) * sizeof(R), a.rows,
                                  dst_on_host ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice, S(stream)));
            if (dst_on_host) GCU(cudaStreamSynchronize(S(stream)));
        });
    });
}

int glide_fill_field(glide_handle h, int field, int level, double value, int restrict_down, void* stream) {
    return guarded([&] {
        dispatch(h, [&](auto& s) {
            using R = std::remove_reference_t<decltype(*s.lv[0].a[0].p)>;
            auto& a = field_arr(s, field, level);
            s.fill(a, R(value), S(stream));
            if (restrict_down)
                for (int l = level; l + 1 < s.n_levels; ++l) s.restrict_field(field, l, S(stream));
        });
    });
}

int glide_restrict_field(glide_handle h, int field, int level, void* stream) {
    return guarded([&] {
        dispatch(h, [&](auto& s) {
            field_arr(s, field, level);
            for (int l = level; l + 1 < s.n_levels; ++l) s.restrict_field(field, l, S(stream));
        });
    });
}

int glide_set_phys(glide_handle h, int level, const glide_phys* p) {
    return guarded([&] {
        if (!p) fail(GLIDE_ERR_ARG, "null phys");
        dispatch(h, [&](auto& s) {
            using R = std::remove_reference_t<decltype(*s.lv[0].a[0].p)>;
            for (int l = 0; l < s.n_levels; ++l) {
                if (level >= 0 && l != level) continue;
                const bool thk_changed = s.lv[l].phys.thklim != p->thklim;
                s.lv[l].phys = *p;
                if (thk_changed) s.fill(s.lv[l].a[GLIDE_GAMMA], R(p->thklim), nullptr);
            }
            if (level >= s.n_levels) fail(GLIDE_ERR_ARG, "level out of range");
            ++s.version;
            GCU(cudaDeviceSynchronize());
        });
    });
}

int glide_get_phys(glide_handle h, int level, glide_phys* p) {
    return guarded([&] {
        if (!p) fail(GLIDE_ERR_ARG, "null phys");
        dispatch(h, [&](auto& s) {
            s.check_level(level);
            *p = s.lv[level].phys;
        });
    });
}

static int which_config(int which) {
    if (which < 0 || which > 2) fail(GLIDE_ERR_ARG, "config selector must be 0 (forward), 1 (adjoint) or 2 (tangent)");
    return which;
}

int glide_set_fas_config(glide_handle h, int which, const glide_fas_config* c) {
    return guarded([&] {
        if (!c) fail(GLIDE_ERR_ARG, "null config");
        dispatch(h, [&](auto& s) {
            s.fas[which_config(which)] = *c;
            ++s.version;
        });
    });
}

int glide_get_fas_config(glide_handle h, int which, glide_fas_config* c) {
    return guarded([&] {
        if (!c) fail(GLIDE_ERR_ARG, "null config");
        dispatch(h, [&](auto& s) { *c = s.fas[which_config(which)]; });
    });
}

int glide_set_vanka_config(glide_handle h, int which, int level, const glide_vanka_config* c) {
    return guarded([&] {
        if (!c) fail(GLIDE_ERR_ARG, "null config");
        dispatch(h, [&](auto& s) {
            const int q = which_config(which);
            if (level >= s.n_levels) fail(GLIDE_ERR_ARG, "level out of range");
            for (int l = 0; l < s.n_levels; ++l)
                if (level < 0 || l == level) s.lv[l].vk[q] = *c;
            ++s.version;
        });
    });
}

int glide_get_vanka_config(glide_handle h, int which, int level, glide_vanka_config* c) {
    return guarded([&] {
        if (!c) fail(GLIDE_ERR_ARG, "null config");
        dispatch(h, [&](auto& s) {
            s.check_level(level);
            *c = s.lv[level].vk[which_config(which)];
        });
    });
}

int glide_set_reference_quirks(glide_handle h, int on) {
    return guarded([&] {
        dispatch(h, [&](auto& s) {
            s.quirks = on ? 1 : 0;
            ++s.version;
        });
    });
}

int glide_set_tuning(glide_handle h, int key, int value) {
    return guarded([&] {
        dispatch(h, [&](auto& s) {
            if (key == GLIDE_TUNE_SWEEP_BLOCKS_PER_SM) {
                if (value < 1 || value > 2) fail(GLIDE_ERR_ARG, "sweep blocks per SM must be 1 or 2");
                s.sweep_blocks_per_sm = value;
            } else if (key == GLIDE_TUNE_MIXED_INNER_VCYCLES) {
                if (value < 1 || value > 16) fail(GLIDE_ERR_ARG, "inner V-cycles must be in [1, 16]");
                s.mixed_inner = value;
            } else if (key == GLIDE_TUNE_FORWARD_METHOD) {
                if (value < 0 || value > 1) fail(GLIDE_ERR_ARG, "forward method must be 0 (FASCD) or 1 (FASCD + Newton)");
                s.forward_method = value;
            } else if (key == GLIDE_TUNE_NEWTON_SWITCH_EXP10) {
                if (value < 0 || value > 15) fail(GLIDE_ERR_ARG, "Newton switch exponent must be in [0, 15]");
                s.newton_switch = std::pow(10.0, -double(value));
            } else if (key == GLIDE_TUNE_TANGENT_VCYCLES) {
                if (value < 1 || value > 16) fail(GLIDE_ERR_ARG, "tangent V-cycles must be in [1, 16]");
                s.tangent_vcycles = value;
            } else if (key == GLIDE_TUNE_TMA_STAGING) {
                if (value < 0 || value > 1) fail(GLIDE_ERR_ARG, "TMA staging must be 0 or 1");
                s.use_tma = value != 0;
            } else if (key == GLIDE_TUNE_TMA_GIVE_UP) {
                if (value < 0 || value > 1) fail(GLIDE_ERR_ARG, "TMA give-up must be 0 or 1");
                s.tma_wait_polls = value ? 0 : kTmaWaitPolls;
            } else if (key == GLIDE_TUNE_REPORT_NOT_CONVERGED) {
                if (value < 0 || value > 1) fail(GLIDE_ERR_ARG, "report-not-converged must be 0 or 1");
                s.report_not_converged = value;
                return;  // no effect on captured graphs
            } else {
                fail(GLIDE_ERR_ARG, "unknown tuning key");
            }
            ++s.version;
        });
    });
}

int glide_set_use_graphs(glide_handle h, int use_graphs) {
    return guarded([&] {
        dispatch(h, [&](auto& s) {
            s.use_graphs = use_graphs ? 1 : 0;
            ++s.version;
        });
    });
}

int glide_set_rhs(glide_handle h, int level, double dt, void* stream) {
    return guarded([&] {
        dispatch(h, [&](auto& s) {
            s.check_level(level);
            s.set_rhs(level, dt, S(stream));
        });
    });
}

int glide_compute_phi(glide_handle h, int level, double relaxation, void* stream) {
    return guarded([&] {
        dispatch(h, [&](auto& s) {
            s.check_level(level);
            s.compute_phi(level, relaxation, S(stream));
        });
    });
}

int glide_residual(glide_handle h, int level, double dt, int flags, double* norms3, void* stream) {
    return guarded([&] {
        dispatch(h, [&](auto& s) {
            s.check_level(level);
            const bool op = flags & GLIDE_OPERATOR_ONLY;
            s.residual(level, dt, !op, (flags & GLIDE_USE_MASK) != 0, (flags & GLIDE_FREEZE_CALVING) != 0,
                       (flags & GLIDE_FREEZE_PHI) != 0, op ? GLIDE_FOP_U : GLIDE_R_U, op ? GLIDE_FOP_V : GLIDE_R_V,
                       op ? GLIDE_FOP_H : GLIDE_R_H, nullptr, norms3 != nullptr, S(stream));
            if (norms3) {
                double nr[4];
                s.read_norms(nr, S(stream));
                for (int q = 0; q < 3; ++q) norms3[q] = nr[q];
            }
        });
    });
}

int glide_vanka_sweep(glide_handle h, int level, double dt, int n, int flags, int* newton_iters, void* stream) {
    return guarded([&] {
        if (n < 0) fail(GLIDE_ERR_ARG, "negative sweep count");
        dispatch(h, [&](auto& s) {
            s.check_level(level);
            s.sweeps(level, dt, n, kGammaArray, (flags & GLIDE_FREEZE_CALVING) != 0,
                     (flags & GLIDE_FREEZE_PHI) != 0, newton_iters, S(stream));
        });
    });
}

int glide_vanka_dump(glide_handle h, int level, double dt, void* J, void* r, void* stream) {
    return guarded([&] {
        if (!J || !r) fail(GLIDE_ERR_ARG, "null output array");
        dispatch(h, [&](auto& s) {
            using RT = std::remove_pointer_t<decltype(s.lv[0].a[0].p)>;
            s.check_level(level);
            s.vanka_dump(level, dt, static_cast<RT*>(J), static_cast<RT*>(r), S(stream));
        });
    });
}

int glide_forward(glide_handle h, double dt, int start_level, glide_stats* stats, void* stream) {
    return guarded([&] {
        dispatch(h, [&](auto& s) {
            s.forward(dt, start_level, stats, S(stream));
            s.report_convergence();
        });
    });
}

int glide_adjoint_residual(glide_handle h, int level, double dt, double* norms3, void* stream) {
    return guarded([&] {
        dispatch(h, [&](auto& s) {
            s.check_level(level);
            s.adj_residual(level, dt, norms3 != nullptr, S(stream));
            if (norms3) {
                double nr[4];
                s.read_norms(nr, S(stream));
                for (int q = 0; q < 3; ++q) norms3[q] = nr[q];
            }
        });
    });
}

int glide_vjp(glide_handle h, int level, double dt, void* stream) {
    return guarded([&] {
        dispatch(h, [&](auto& s) {
            s.check_level(level);
            s.vjp_into(level, dt, false, GLIDE_VJP_U, GLIDE_VJP_V, GLIDE_VJP_H, S(stream));
        });
    });
}

int glide_jvp(glide_handle h, int level, double dt, int reference_rows, int flags, void* stream) {
    return guarded([&] {
        dispatch(h, [&](auto& s) {
            s.check_level(level);
            using SolverT = std::remove_reference_t<decltype(s)>;
            typename SolverT::Lin L = SolverT::tan_sys();
            L.x[0] = GLIDE_VAR_U; L.x[1] = GLIDE_VAR_V; L.x[2] = GLIDE_VAR_H;
            const int out[3] = {GLIDE_JVP_U, GLIDE_JVP_V, GLIDE_JVP_H};
            if (flags & ~(GLIDE_USE_MASK | GLIDE_FREEZE_CALVING))
                fail(GLIDE_ERR_ARG, "glide_jvp flags: only GLIDE_USE_MASK and GLIDE_FREEZE_CALVING apply");
            s.lin_op(level, dt, L, out, nullptr, false, false, reference_rows != 0, S(stream), flags);
        });
    });
}

int glide_adjoint_sweep(glide_handle h, int level, double dt, int n, void* stream) {
    return guarded([&] {
        if (n < 0) fail(GLIDE_ERR_ARG, "negative sweep count");
        dispatch(h, [&](auto& s) {
            s.check_level(level);
            s.ensure_blocks();
            s.adj_sweeps(level, dt, n, S(stream));
        });
    });
}

int glide_gradients(glide_handle h, int level, double dt, int grad_mask, void* stream) {
    return guarded([&] {
        dispatch(h, [&](auto& s) {
            s.check_level(level);
            s.gradients(level, dt, grad_mask, S(stream));
        });
    });
}

int glide_launch_count(glide_handle h, long long* count) {
    return guarded([&] {
        if (!count) fail(GLIDE_ERR_ARG, "null count");
        dispatch(h, [&](auto& s) { *count = s.launches; });
    });
}

int glide_block_smoother_part(glide_handle h, int level, double dt, int adjoint, int part, void* stream) {
    return guarded([&] {
        if (part < 0 || part > 1) fail(GLIDE_ERR_ARG, "part must be 0 (factorisation) or 1 (sweep)");
        dispatch(h, [&](auto& s) {
            s.check_level(level);
            s.block_part(level, dt, adjoint != 0, part, S(stream));
        });
    });
}

int glide_alg_bytes(glide_handle h, double* bytes) {
    return guarded([&] {
        if (!bytes) fail(GLIDE_ERR_ARG, "null output");
        dispatch(h, [&](auto& s) { *bytes = s.alg_bytes; });
    });
}

int glide_backward(glide_handle h, double dt, int start_level, int grad_mask, glide_stats* stats, void* stream) {
    return guarded([&] {
        dispatch(h, [&](auto& s) {
            s.backward(dt, start_level, grad_mask, stats, S(stream));
            s.report_convergence();
        });
    });
}

int glide_vcycle(glide_handle h, int which, int level, int finest, double dt, void* stream) {
    return guarded([&] {
        if (which != 0 && which != 1) fail(GLIDE_ERR_ARG, "which must be 0 (FASCD) or 1 (adjoint)");
        dispatch(h, [&](auto& s) {
            s.check_level(level);
            if (which == 0) {
                s.check_quirks();
                s.vcycle(level, finest != 0, dt, S(stream));
            } else {
                s.ensure_blocks();
                s.adj_vcycle(level, finest != 0, dt, S(stream));
            }
        });
    });
}

int glide_transfer(int op, int dtype, int ny_fine, int nx_fine, const void* src, int ld_src, void* dst, int ld_dst,
                   void* stream) {
    return guarded([&] {
        if (!src || !dst) fail(GLIDE_ERR_ARG, "null array");
        if (op < GLIDE_RESTRICT_VFACET || op > GLIDE_PROLONG_HFACET_AS_VFACET_BILINEAR)
            fail(GLIDE_ERR_ARG, "unknown transfer op");
        if (dtype != GLIDE_F64 && dtype != GLIDE_F32) fail(GLIDE_ERR_ARG, "dtype must be GLIDE_F64 or GLIDE_F32");
        if (ny_fine < 2 || nx_fine < 2 || (ny_fine & 1) || (nx_fine & 1))
            fail(GLIDE_ERR_SHAPE, "fine cell counts must be even and >= 2");
        if (op >= GLIDE_PROLONG_HFACET_AS_VFACET_INJECTION && ny_fine != nx_fine)
            fail(GLIDE_ERR_SHAPE, "the u-face prolongation of v-face memory needs a square grid");
        const int nyc = ny_fine / 2, nxc = nx_fine / 2;
        // (rows, cols) of the fine and coarse arrays of this field's kind
        int fr = ny_fine, fc = nx_fine, cr = nyc, cc = nxc;
        const bool ufaces = op == GLIDE_RESTRICT_VFACET || op == GLIDE_PROLONG_VFACET_INJECTION ||
                            op == GLIDE_PROLONG_VFACET_BILINEAR;
        const bool vfaces = op == GLIDE_RESTRICT_HFACET || op == GLIDE_PROLONG_HFACET_INJECTION ||
                            op == GLIDE_PROLONG_HFACET_BILINEAR || op >= GLIDE_PROLONG_HFACET_AS_VFACET_INJECTION;
        if (ufaces) ++fc, ++cc;
        if (vfaces) ++fr, ++cr;
        const bool restrict_op = op <= GLIDE_RESTRICT_CELL_VAR;
        const int sr = restrict_op ? fr : cr, sc = restrict_op ? fc : cc;
        const int dr = restrict_op ? cr : fr, dc = restrict_op ? cc : fc;
        if (ld_src < sc || ld_dst < dc) fail(GLIDE_ERR_ARG, "leading dimension smaller than the row length");
        auto run = [&](auto* s) {
            using R = std::remove_const_t<std::remove_pointer_t<decltype(s)>>;
            Arr<R> a{const_cast<R*>(s), sr, sc, ld_src}, b{static_cast<R*>(dst), dr, dc, ld_dst};
            k_transfer<R><<<dim3((dc + 255) / 256, dr), 256, 0, S(stream)>>>(a, b, op, ny_fine, nx_fine);
            check_launch("k_transfer");
        };
        if (dtype == GLIDE_F64) run(static_cast<const double*>(src));
        else run(static_cast<const float*>(src));
    });
}

int glide_group_create(const glide_handle* members, int n, glide_group* out) {
    return guarded([&] {
        if (!out) fail(GLIDE_ERR_ARG, "out is null");
        *out = nullptr;
        if (!members || n <= 0) fail(GLIDE_ERR_ARG, "a group needs at least one member");
        if (n > kGroupControlThreads) fail(GLIDE_ERR_ARG, "too many members");
        for (int k = 0; k < n; ++k) {
            if (!members[k] || !members[k]->impl) fail(GLIDE_ERR_ARG, "null member handle");
            for (int q = 0; q < k; ++q)
                if (members[q] == members[k]) fail(GLIDE_ERR_ARG, "a handle appears twice in the group");
            if (members[k]->impl->dtype != members[0]->impl->dtype)
                fail(GLIDE_ERR_ARG, "group members must share one dtype");
        }
        auto g = std::make_unique<glide_group_s>();
        if (members[0]->impl->dtype == GLIDE_F64) {
            std::vector<Solver<double>*> v;
            for (int k = 0; k < n; ++k) {
                auto* m = static_cast<Solver<double>*>(members[k]->impl.get());
                if (m->lo) fail(GLIDE_ERR_STATE, "mixed-precision hierarchies have no grouped form");
                v.push_back(m);
            }
            g->impl = std::make_unique<GroupRun<double>>(std::move(v));
        } else {
            std::vector<Solver<float>*> v;
            for (int k = 0; k < n; ++k) v.push_back(static_cast<Solver<float>*>(members[k]->impl.get()));
            g->impl = std::make_unique<GroupRun<float>>(std::move(v));
        }
        *out = g.release();
    });
}

int glide_group_destroy(glide_group g) {
    return guarded([&] { delete g; });
}

int glide_group_forward(glide_group g, double dt, int start_level, glide_stats* stats, void* stream) {
    return guarded([&] {
        if (!g || !g->impl) fail(GLIDE_ERR_ARG, "null group");
        g->impl->forward(dt, start_level, stats, S(stream));
    });
}

int glide_group_backward(glide_group g, double dt, int start_level, int grad_mask, glide_stats* stats,
                         void* stream) {
    return guarded([&] {
        if (!g || !g->impl) fail(GLIDE_ERR_ARG, "null group");
        g->impl->backward(dt, start_level, grad_mask, stats, S(stream));
    });
}

int glide_group_set_tuning(glide_group g, int key, int value) {
    return guarded([&] {
        if (!g || !g->impl) fail(GLIDE_ERR_ARG, "null group");
        if (key == GLIDE_GROUP_TUNE_WAVES) {
            if (value < 0 || value > 64) fail(GLIDE_ERR_ARG, "waves must lie in [0, 64]");
            g->impl->waves = value;
            g->impl->invalidate();
        } else if (key == GLIDE_GROUP_TUNE_SPOIL_MAPS) {
            if (value != 0 && value != 1) fail(GLIDE_ERR_ARG, "spoil_maps must be 0 or 1");
            g->impl->spoil_maps = value;
            g->impl->invalidate();
        } else {
            fail(GLIDE_ERR_ARG, "unknown group tuning key");
        }
    });
}

int glide_group_counters(glide_group g, long long* launches, int* shape) {
    return guarded([&] {
        if (!g || !g->impl) fail(GLIDE_ERR_ARG, "null group");
        if (launches) *launches = g->impl->launches;
        if (shape)
            for (int q = 0; q < 4; ++q) shape[q] = g->impl->shape[q];
    });
}

}  // extern "C"
