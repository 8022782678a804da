// solver.cu - host side of the B200 cavity solver and its C ABI (cavity_solver.h).
//
// One `Solver<T>` owns one cavity: its fields in HBM, a CUDA stream, and two instantiated CUDA graphs of a
// whole time step (one per state parity, since the step writes the next state into the other buffer set).
// A step is one graph launch: 1 + 3 x 4 kernels plus, per stage, a conditional while-node whose body is one
// pressure pass (6 transform launches and a residual); the residual's last block decides on the device
// whether another pass runs.  The host waits once per step, to read the 200-byte control block that holds
// the clock, the report and any error.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <map>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <vector>

#include "cavity_solver.h"
#include "kernels.cuh"
#include "fdm.cuh"
#include "tc_gemm.cuh"
#include "sweep.cuh"
#include "sweep_march.cuh"
#include "sweep_tile.cuh"
#include "sweep_pair.cuh"
#include "outputs.cuh"
#include "setup.h"

namespace cavity {

[[noreturn]] static void fail(const std::string& m) { throw std::runtime_error(m); }
static void check(cudaError_t e) {
    if (e != cudaSuccess) fail(std::string("CUDA error: ") + cudaGetErrorString(e));
}
static unsigned int blocks_for(long long n) { return (unsigned int)((n + kThreads - 1) / kThreads); }

// ------------------------------------------------------------------------------------------ device memory
// Device memory of one solver: a block reserved up front (one cudaMalloc, zero-filled once) from which the
// arrays are carved at 256-byte alignment, and separate zero-filled allocations for anything beyond it.  One
// allocation instead of dozens keeps creating and destroying a solver cheap when many come and go (serving).
class DeviceArena {
public:
    ~DeviceArena() { release(); }
    void reserve(size_t bytes) {
        bytes = (bytes + 255) / 256 * 256;
        check(cudaMalloc(&block_, bytes));
        check(cudaMemset(block_, 0, bytes));
        ptrs_.push_back(block_);
        cap_ = bytes;
        used_ = 0;
    }
    template <class T> T* alloc(long long n) {
        const size_t bytes = sizeof(T) * (size_t)std::max(n, 1LL);
        bytes_ += bytes;
        const size_t need = (bytes + 255) / 256 * 256;
        if (block_ && used_ + need <= cap_) {
            void* p = static_cast<char*>(block_) + used_;
            used_ += need;
            return (T*)p;
        }
        void* p = nullptr;
        check(cudaMalloc(&p, bytes));
        check(cudaMemset(p, 0, bytes));
        ptrs_.push_back(p);
        return (T*)p;
    }
    void release() {
        for (void* p : ptrs_) cudaFree(p);
        ptrs_.clear();
        block_ = nullptr;
        cap_ = used_ = 0;
        bytes_ = 0;
    }
    long long bytes() const { return bytes_; }
private:
    std::vector<void*> ptrs_;
    void* block_ = nullptr;
    size_t cap_ = 0, used_ = 0;
    long long bytes_ = 0;
};

static long long estimate_bytes(const CavityConfig& c, int precision);

// ------------------------------------------------------------------------------------------ autotuner cache
// Launch shapes chosen by timing (Solver::autotune), per grid size, stretching and precision form: the z-chunk
// count of the march sweep and the FP64 transform tile.  Neither changes the arithmetic of a step.  Kept for the
// process and, when CAVITY_TUNE_FILE names a file, read from it once and appended to it.
struct Tuning {
    int chunks = 0;       // march sweep z-chunks (0: the device-filling rule)
    int dgemm = 0;        // FP64 transform tile, 32 or 64 (0: the size rule)
    int fused = -1;       // FP64 pass form (PassForm: 0 six launches, 1 one cooperative launch, 2 paired), -1 by size
    int sweep = -1;       // momentum sweep kernel (SweepKind; -1: not chosen)
    float ms = 0;         // measured step time of the choice
};
static std::string tune_key(const CavityConfig& c, int precision) {
    char k[160];
    std::snprintf(k, sizeof k, "%d %d %d %d %.17g %.17g %d", c.nx, c.ny, c.nz, c.grid_stretch,
                  c.grid_stretch ? c.grid_dx_wall : 0.0, c.grid_stretch ? c.grid_max_aspect : 0.0, precision);
    return k;
}
static std::mutex g_tune_mutex;
static std::map<std::string, Tuning> g_tune;
static bool g_tune_file_read = false;
static const char* tune_file() {
    const char* f = std::getenv("CAVITY_TUNE_FILE");
    return f && *f ? f : nullptr;
}
// the cached tuning of a key, if any (call with g_tune_mutex held)
static const Tuning* tune_lookup(const std::string& key) {
    if (!g_tune_file_read) {
        g_tune_file_read = true;
        if (const char* f = tune_file()) {
            if (FILE* fp = std::fopen(f, "r")) {
                char line[256];
                while (std::fgets(line, sizeof line, fp)) {
                    const char* bar = std::strchr(line, '|');
                    Tuning t;
                    if (!bar || std::sscanf(bar + 1, "%d %d %d %d %f", &t.chunks, &t.dgemm, &t.fused, &t.sweep, &t.ms) != 5)
                        continue;
                    std::string k(line, bar - line);
                    while (!k.empty() && k.back() == ' ') k.pop_back();
                    g_tune[k] = t;
                }
                std::fclose(fp);
            }
        }
    }
    auto it = g_tune.find(key);
    return it == g_tune.end() ? nullptr : &it->second;
}
static void tune_store(const std::string& key, const Tuning& t) {
    std::lock_guard<std::mutex> lock(g_tune_mutex);
    tune_lookup(key);
    g_tune[key] = t;
    if (const char* f = tune_file()) {
        if (FILE* fp = std::fopen(f, "a")) {
            std::fprintf(fp, "%s | %d %d %d %d %.6f\n", key.c_str(), t.chunks, t.dgemm, t.fused, t.sweep, t.ms);
            std::fclose(fp);
        }
    }
}

class SolverBase {
public:
    virtual ~SolverBase() {}
    virtual void initialize(const double* v, const double* w) = 0;
    virtual void step_async(int count) = 0;
    virtual void sync(CavityReport* r) = 0;
    virtual void report(CavityReport* r) = 0;
    virtual void kick(const double* const n[3], double amp, int passes) = 0;
    virtual void diagnostics(CavityDiagnostics* d) = 0;
    virtual void grid(int axis, double* faces, double* centres) = 0;
    virtual void get_field(int field, void* out) = 0;
    virtual void get_field_f64(int field, double* out) = 0;
    virtual void set_field(int field, const void* in) = 0;
    virtual void set_clock(double t, long long steps, double last_dt) = 0;
    virtual void probes(float* out) = 0;
    virtual void add_statistics(double weight, double* centreline) = 0;
    virtual void get_statistics(double* sums) = 0;
    virtual void step_outputs_async(int count, int statistics) = 0;
    virtual int sync_outputs(CavityReport* r, float* probes, int max_steps) = 0;
    virtual long long checkpoint_bytes() const = 0;
    virtual void checkpoint_save(void* dst, int device) = 0;
    virtual void checkpoint_load(const void* src, int device) = 0;
    virtual void set_statistics(const double* sums) = 0;
    virtual void midplane(float* out) = 0;
    virtual void q_volume(int colour_w, float* q, float* colour) = 0;
    virtual long long device_bytes() const = 0;
    virtual void time_steps(int warmup, int steps, int flush, float* ms, float* kms) = 0;
    virtual void kernel_times(double* ms) const = 0;
    virtual int kernels_per_step(int passes) const = 0;
    virtual long long pressure_passes() const = 0;
    virtual void autotune(int steps, int* chunks, int* dgemm_tile, int* fused, float* ms) = 0;
    void step(CavityReport* r) {
        step_async(1);
        sync(r);
    }
};

// ------------------------------------------------------------------------------------------ the solver
template <class T> class Batch;

template <class T> class Solver : public SolverBase {
    friend class Batch<T>;
    // tile of the shared-memory sweep: 32 x TY x TZ cells (about 113 KB of shared memory in FP64, 85 KB in FP32)
    static constexpr int kTileTY = sizeof(T) == 8 ? 4 : 8;
    static constexpr int kTileTZ = 4;
    static constexpr int kTileNT = sizeof(T) == 8 ? 256 : 512;     // threads: registers allow 512 in FP32
    using TileG = TileGeom<kTileTY, kTileTZ, kTileNT>;
    // the FP32 tile sweep with two cells per thread in packed arithmetic (sweep_pair.cuh): the same tile, 256 threads
    static constexpr int kPairNT = 256;
    using PairG = TileGeom<kTileTY, kTileTZ, kPairNT, true>;
    // the z-march sweep (sweep_march.cuh): 32 x 8 columns of cells per CTA
    static constexpr int kMarchTX = 32, kMarchTY = 8;
    using MarchG = MarchGeom<kMarchTX, kMarchTY>;

public:
    explicit Solver(const CavityConfig& cfg) : c_(cfg) {
        const std::string bad = check_config(c_);
        if (!bad.empty()) fail(bad);
        nx_ = c_.nx; ny_ = c_.ny; nz_ = c_.nz;
        n_cell_ = (long long)nx_ * ny_ * nz_;
        for (int k = 0; k < 3; k++) size_[k] = (long long)(nx_ + (k == 0)) * (ny_ + (k == 1)) * (nz_ + (k == 2));
        max_face_ = std::max(size_[0], std::max(size_[1], size_[2]));
        ax_[0] = make_axis_grid(c_, nx_, c_.length);
        ax_[1] = make_axis_grid(c_, ny_, c_.length);
        ax_[2] = make_axis_grid(c_, nz_, nz_ * (c_.lz / nz_));
        volume_ = ax_[0].length * ax_[1].length * ax_[2].length;
        check(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
        check(cudaStreamCreateWithFlags(&body_stream_, cudaStreamNonBlocking));
        setup_params();
        arena_.reserve((size_t)estimate_bytes(c_, sizeof(T) == 8 ? 0 : 1));
        {
            // Mixed form: FDM transforms on the tcgen05 tensor cores (3xTF32) from 128^3 cells up, FP64 DMMA
            // transforms below.  FP32 transforms need two refinement passes where FP64 ones need one, which
            // only pays once the transforms are large; CAVITY_FDM=tc or =dmma forces either.  The tensor-core
            // kernel's float4 row loads need nx % 4 == 0.
            const char* f = std::getenv("CAVITY_FDM");
            const std::string fdm = f ? f : "";
            const bool want = fdm == "tc" || (fdm != "dmma" && n_cell_ >= (1LL << 21));
            tc_fdm_ = sizeof(T) == 4 && nx_ % 4 == 0 && want;
        }
        allocate();
        upload_tables();
        build_graphs();
        {
            std::lock_guard<std::mutex> lock(g_tune_mutex);
            if (const Tuning* t = tune_lookup(tune_key(c_, sizeof(T) == 8 ? 0 : 1))) tune_ = *t;
        }
        if (tune_.sweep >= 0 && !sweep_forced_) sweep_kind_ = tune_.sweep;
        if (const char* a = std::getenv("CAVITY_AUTOTUNE")) auto_tune_ = a[0] == '1';
        check(cudaStreamSynchronize(stream_));
    }
    ~Solver() override {
        for (int s = 0; s < 2; s++) {
            if (exec_[s]) cudaGraphExecDestroy(exec_[s]);
            if (graph_[s]) cudaGraphDestroy(graph_[s]);
            if (texec_[s]) cudaGraphExecDestroy(texec_[s]);
            if (tgraph_[s]) cudaGraphDestroy(tgraph_[s]);
        }
        for (cudaEvent_t& e : kev_) if (e) cudaEventDestroy(e);
        if (stream_) cudaStreamSynchronize(stream_);
        arena_.release();
        if (flush_) cudaFree(flush_);
        if (ring_host_) cudaFreeHost(ring_host_);
        if (tail_host_) cudaFreeHost(tail_host_);
        if (stream_) cudaStreamDestroy(stream_);
        if (body_stream_) cudaStreamDestroy(body_stream_);
    }

    // -------------------------------------------------------------------------------- ABI operations
    void initialize(const double* v_noise, const double* w_noise) override {         // backend.cu:1075-1088
        probes_fresh_ = false;
        const double* src[3] = {nullptr, v_noise, w_noise};
        for (int k = 0; k < 3; k++) {
            if (src[k]) check(cudaMemcpyAsync(dstage_[0], src[k], sizeof(double) * size_[k], cudaMemcpyHostToDevice, stream_));
            noise_to_field_kernel<T><<<blocks_for(size_[k]), kThreads, 0, stream_>>>(src[k] ? dstage_[0] : nullptr, M_[par_][k], size_[k]);
        }
        T* m[3] = {M_[par_][0], M_[par_][1], M_[par_][2]};
        T* u[3] = {U_[par_][0], U_[par_][1], U_[par_][2]};
        project(m, PHI_[par_], u);
        hc_.t = 0; hc_.steps = 0; hc_.last_dt = 0; hc_.hist_count = 0; hc_.have_prev = 0;
        push_control();
        check(cudaStreamSynchronize(stream_));
    }

    void step_async(int count) override {
        if (auto_tune_ && tune_.ms == 0 && pending_.empty()) autotune(6, nullptr, nullptr, nullptr, nullptr);
        ensure_graphs(false);
        if (pending_.empty()) steps_before_ = hc_.steps;
        if (!tail_host_) {
            const size_t off = 256 * ((sizeof(Control) + 255) / 256);
            check(cudaHostAlloc(&tail_host_, off + sizeof(float) * 16, cudaHostAllocMapped));
            check(cudaHostGetDevicePointer(&tail_dev_, tail_host_, 0));
        }
        probes_fresh_ = false;
        for (int i = 0; i < count; i++) {
            if (eager_) enqueue_step(par_, false, true);
            else check(cudaGraphLaunch(exec_[par_], stream_));
            // the parity flips only when the step succeeds; sync() checks that for the queued steps
            pending_.push_back(par_);
            par_ ^= 1;
            char* d = static_cast<char*>(tail_dev_);
            step_tail_kernel<T><<<1, 32, 0, stream_>>>(out_args(), probe_cells_, c_.n_probes,
                                                       reinterpret_cast<float*>(d + 256 * ((sizeof(Control) + 255) / 256)),
                                                       ctrl_, reinterpret_cast<Control*>(d));
        }
        tail_queued_ = true;
    }
    void sync(CavityReport* r) override {
        check(cudaStreamSynchronize(stream_));
        if (tail_queued_) std::memcpy(&hc_, tail_control(), sizeof hc_);      // written by the last step's tail
        else pull_control();
        const bool tail = tail_queued_;
        tail_queued_ = false;
        probes_fresh_ = false;
        const size_t queued = pending_.size();
        const std::vector<int> pending_copy = pending_;
        pending_.clear();
        if (hc_.error) {
            // steps before the failed one committed; the failed step left the state buffers of its parity
            // untouched and every later queued step skipped its work
            const long long ok = hc_.steps - steps_before_;
            par_ = (ok >= 0 && ok < (long long)queued) ? pending_copy[ok] : par_;
            const int code = hc_.error;
            hc_.error = kOk;
            push_control();
            check(cudaStreamSynchronize(stream_));
            raise_error(code);
        }
        check(cudaGetLastError());
        probes_fresh_ = tail && !pending_copy.empty();
        if (r) report(r);
    }
    void report(CavityReport* r) override {
        r->steps = hc_.steps; r->time = hc_.t; r->dt = hc_.last_dt; r->cfl = hc_.last_cfl;
        r->phi_rel = hc_.phi_rel; r->dt_reason = hc_.dt_reason; r->phi_passes = hc_.phi_passes;
    }

    void kick(const double* const noise[3], double amp, int passes) override {        // backend.cu:958-978
        probes_fresh_ = false;
        const int S = par_, X2 = par_ ^ 1;
        for (int k = 0; k < 3; k++) {
            const int sx = nx_ + (k == 0), sy = ny_ + (k == 1), sz = nz_ + (k == 2);
            check(cudaMemcpyAsync(dstage_[0], noise[k], sizeof(double) * size_[k], cudaMemcpyHostToDevice, stream_));
            double* a = dstage_[0];
            double* b = dstage_[1];
            for (int p = 0; p < std::max(1, passes); p++)
                for (int axis = 2; axis >= 0; axis--) {
                    smooth_kernel<<<blocks_for(size_[k]), kThreads, 0, stream_>>>(a, b, axis, sx, sy, sz);
                    std::swap(a, b);
                }
            sumsq_kernel<<<blocks_for(size_[k]), kThreads, 0, stream_>>>(a, size_[k], slots_, partial_, out_counters_);
            add_noise_kernel<T><<<blocks_for(size_[k]), kThreads, 0, stream_>>>(U_[S][k], a, slots_, amp * c_.u_lid,
                                                                               size_[k], M0_[k]);
        }
        // project the disturbed velocity (scratch potential; the state potential is unchanged)
        T* tmp[3] = {M0_[0], M0_[1], M0_[2]};
        T* nu[3] = {U_[X2][0], U_[X2][1], U_[X2][2]};
        project(tmp, PHI_[2], nu);
        for (int k = 0; k < 3; k++)
            kick_update_kernel<T><<<blocks_for(size_[k]), kThreads, 0, stream_>>>(M_[S][k], U_[S][k], U_[X2][k], size_[k]);
        check(cudaStreamSynchronize(stream_));
        check(cudaGetLastError());
    }

    void diagnostics(CavityDiagnostics* d) override {                                  // backend.cu:1096-1129
        OutArgs<T> a = out_args();
        const T lidv = (T)lid_speed_host(hc_.t);
        cell_diag_kernel<T><<<blocks_for(n_cell_), kThreads, 0, stream_>>>(a, lidv);
        for (int k = 0; k < 3; k++)
            max_abs_kernel<T><<<blocks_for(size_[k]), kThreads, 0, stream_>>>(a, k, size_[k], partial_ + 4 * partial_blocks_);
        double slots[kNumSlots];
        check(cudaMemcpyAsync(slots, slots_, sizeof slots, cudaMemcpyDeviceToHost, stream_));
        check(cudaStreamSynchronize(stream_));
        d->kinetic_energy = slots[kSlotKE] / volume_;
        d->enstrophy = 0.5 * slots[kSlotEns] / volume_;
        d->div_rms = std::sqrt(slots[kSlotDiv2] / volume_);
        double umax = 0;
        for (int k = 0; k < 3; k++) umax = std::max(umax, slots[kSlotUmax0 + k]);
        d->umax = umax;
        d->cfl_rate = hc_.cfl_rate;
        double best = -1;
        int best_comp = 0;
        long long best_i = 0;
        for (int k = 0; k < 3; k++) {
            const double val = slots[kSlotGauge0 + k];
            if (val > best) { best = val; best_comp = k; best_i = (long long)slots[kSlotGaugeIdx0 + k]; }
        }
        const int sx = nx_ + (best_comp == 0), sy = ny_ + (best_comp == 1);
        const int ix = (int)(best_i % sx), iy = (int)((best_i / sx) % sy);
        d->gauge_ratio = best / std::max(umax, 1e-30);
        d->gauge_x = (best_comp == 0 ? ax_[0].face[ix] : ax_[0].centre[std::min(ix, nx_ - 1)]) / c_.length;
        d->gauge_y = (best_comp == 1 ? ax_[1].face[iy] : ax_[1].centre[std::min(iy, ny_ - 1)]) / c_.length;
    }

    void grid(int axis, double* faces, double* centres) override {
        if (axis < 0 || axis > 2) fail("axis must be 0, 1 or 2");
        std::copy(ax_[axis].face.begin(), ax_[axis].face.end(), faces);
        std::copy(ax_[axis].centre.begin(), ax_[axis].centre.end(), centres);
    }

    void get_field(int field, void* out) override {                                   // backend.cu:1139-1146
        if (field < 0 || field > 6) fail("field must be 0..6");
        if (field == 6) {
            check(cudaMemcpyAsync(out, PHI_[par_], sizeof(double) * n_cell_, cudaMemcpyDeviceToHost, stream_));
        } else {
            const int k = field % 3;
            const T* src = field < 3 ? U_[par_][k] : M_[par_][k];
            convert_kernel<T, float><<<blocks_for(size_[k]), kThreads, 0, stream_>>>(src, fstage_, size_[k]);
            check(cudaMemcpyAsync(out, fstage_, sizeof(float) * size_[k], cudaMemcpyDeviceToHost, stream_));
        }
        check(cudaStreamSynchronize(stream_));
    }
    void get_field_f64(int field, double* out) override {
        if (field < 0 || field > 6) fail("field must be 0..6");
        if (field == 6) {
            check(cudaMemcpyAsync(out, PHI_[par_], sizeof(double) * n_cell_, cudaMemcpyDeviceToHost, stream_));
        } else {
            const int k = field % 3;
            const T* src = field < 3 ? U_[par_][k] : M_[par_][k];
            convert_kernel<T, double><<<blocks_for(size_[k]), kThreads, 0, stream_>>>(src, dstage_[0], size_[k]);
            check(cudaMemcpyAsync(out, dstage_[0], sizeof(double) * size_[k], cudaMemcpyDeviceToHost, stream_));
        }
        check(cudaStreamSynchronize(stream_));
    }
    void set_field(int field, const void* in) override {                              // backend.cu:1147-1155
        probes_fresh_ = false;
        if (field < 0 || field > 6) fail("field must be 0..6");
        if (field == 6) {
            check(cudaMemcpyAsync(PHI_[par_], in, sizeof(double) * n_cell_, cudaMemcpyHostToDevice, stream_));
        } else {
            const int k = field % 3;
            T* dst = field < 3 ? U_[par_][k] : M_[par_][k];
            check(cudaMemcpyAsync(fstage_, in, sizeof(float) * size_[k], cudaMemcpyHostToDevice, stream_));
            convert_kernel<float, T><<<blocks_for(size_[k]), kThreads, 0, stream_>>>(fstage_, dst, size_[k]);
        }
        hc_.hist_count = 0;
        hc_.have_prev = 0;
        push_control();
        update_cfl();
        check(cudaStreamSynchronize(stream_));
        pull_control();
    }
    // ---- queued steps with their per-step outputs on the device: after each step the probe values go into a
    // ring of pinned, mapped host memory (written by the probe kernel, no copy), and optionally the mid-span
    // statistics accumulate with that step's dt (backend.cu:507-517); nothing waits for the host until
    // sync_outputs.  The reference's run script instead calls solver_step, solver_probes and
    // solver_add_statistics per step, each a blocking round trip.
    static constexpr int kRingSteps = 4096;
    void step_outputs_async(int count, int statistics) override {
        ensure_graphs(false);
        const int np = c_.n_probes;
        if (np > 0 && !ring_host_) {
            check(cudaHostAlloc((void**)&ring_host_, sizeof(float) * 2 * np * kRingSteps, cudaHostAllocMapped));
            check(cudaHostGetDevicePointer((void**)&ring_dev_, ring_host_, 0));
        }
        if (ring_n_ + count > kRingSteps) fail("queued outputs: at most 4096 steps between syncs");
        for (int i = 0; i < count; i++) {
            step_async(1);
            if (np > 0) {
                probes_kernel<T><<<1, 32, 0, stream_>>>(out_args(), probe_cells_, np, ring_dev_ + (size_t)ring_n_ * 2 * np);
                ring_n_++;
            }
            if (statistics)
                statistics_kernel<T><<<blocks_for((long long)nx_ * ny_ + nx_), kThreads, 0, stream_>>>(out_args(), 0.0, ctrl_,
                                                                                                   stats_, line_);
        }
        check(cudaGetLastError());
    }
    // waits for the queued steps; copies the probe values of up to max_steps of them (2 n_probes floats each,
    // in order) and returns how many steps they cover
    int sync_outputs(CavityReport* r, float* probes, int max_steps) override {
        const int queued = ring_n_;
        ring_n_ = 0;
        sync(r);
        const int n = std::min(queued, std::max(max_steps, 0));
        if (n > 0 && probes) std::memcpy(probes, ring_host_, sizeof(float) * 2 * c_.n_probes * n);
        return n;
    }

    // ---- checkpoints: the whole state that decides the following steps, including what the reference drops
    // on restart (backend.cu:1153): the potential-increment history and its times, the dt lag and the CFL rate
    // (all in the control block), plus the statistics sums.  Layout: header, control block, u, m, phi, the
    // four history buffers, statistics; each part 256-byte aligned.
    struct CkHeader {
        unsigned long long magic;
        int nx, ny, nz, field_bytes;
        unsigned long long config_key;      // config_key(): the settings that decide how the state evolves
    };
    // FNV-1a over the settings that decide the next steps (everything but the probe positions), field by
    // field so that struct padding never enters it
    unsigned long long config_key() const {
        unsigned long long h = 1469598103934665603ull;
        auto mix = [&](const void* p, size_t n) {
            const unsigned char* b = static_cast<const unsigned char*>(p);
            for (size_t i = 0; i < n; i++) h = (h ^ b[i]) * 1099511628211ull;
        };
        const int ints[] = {c_.nx, c_.ny, c_.nz, c_.lid_shaped, c_.impulse_order, c_.adaptive_dt, c_.dt_lag,
                            c_.phi_extrapolate, c_.fdm_max_passes, c_.grid_stretch};
        const double dbls[] = {c_.length, c_.u_lid, c_.nu, c_.lz, c_.lid_ramp_t, c_.reinit_r, c_.impulse_order4_ramp,
                               c_.grid_dx_wall, c_.grid_max_aspect, c_.dt_fixed, c_.dt_max, c_.cfl_target,
                               c_.diffusion_limit, c_.fdm_rtol};
        mix(ints, sizeof ints);
        mix(dbls, sizeof dbls);
        return h;
    }
    static constexpr unsigned long long kCkMagic = 0x43415654594b5031ull;
    struct CkLayout {
        size_t ctrl, u[3], m[3], phi, hist[4], stats, total;
    };
    CkLayout ck_layout() const {
        CkLayout L;
        size_t o = 256;
        auto take = [&](size_t bytes) { const size_t at = o; o += (bytes + 255) / 256 * 256; return at; };
        L.ctrl = take(sizeof(Control));
        for (int k = 0; k < 3; k++) L.u[k] = take(sizeof(T) * size_[k]);
        for (int k = 0; k < 3; k++) L.m[k] = take(sizeof(T) * size_[k]);
        L.phi = take(sizeof(double) * n_cell_);
        for (int k = 0; k < 4; k++) L.hist[k] = take(sizeof(double) * n_cell_);
        L.stats = take(sizeof(double) * 6 * nx_ * ny_);
        L.total = o;
        return L;
    }
    long long checkpoint_bytes() const override { return (long long)ck_layout().total; }
    void checkpoint_save(void* dst, int device) override {
        if (!pending_.empty()) fail("checkpoint: steps are queued; sync first");
        const CkLayout L = ck_layout();
        const cudaMemcpyKind kind = device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
        char* d = static_cast<char*>(dst);
        const CkHeader h{kCkMagic, nx_, ny_, nz_, (int)sizeof(T), config_key()};
        check(cudaMemcpyAsync(d, &h, sizeof h, device ? cudaMemcpyHostToDevice : cudaMemcpyHostToHost, stream_));
        check(cudaMemcpyAsync(d + L.ctrl, ctrl_, sizeof(Control), kind, stream_));
        for (int k = 0; k < 3; k++) {
            check(cudaMemcpyAsync(d + L.u[k], U_[par_][k], sizeof(T) * size_[k], kind, stream_));
            check(cudaMemcpyAsync(d + L.m[k], M_[par_][k], sizeof(T) * size_[k], kind, stream_));
        }
        check(cudaMemcpyAsync(d + L.phi, PHI_[par_], sizeof(double) * n_cell_, kind, stream_));
        for (int k = 0; k < 4; k++) check(cudaMemcpyAsync(d + L.hist[k], hist_[k], sizeof(double) * n_cell_, kind, stream_));
        check(cudaMemcpyAsync(d + L.stats, stats_, sizeof(double) * 6 * nx_ * ny_, kind, stream_));
        check(cudaStreamSynchronize(stream_));
    }
    void checkpoint_load(const void* src, int device) override {
        probes_fresh_ = false;
        if (!pending_.empty()) fail("checkpoint: steps are queued; sync first");
        const CkLayout L = ck_layout();
        const cudaMemcpyKind kind = device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
        const char* d = static_cast<const char*>(src);
        CkHeader h;
        check(cudaMemcpy(&h, d, sizeof h, device ? cudaMemcpyDeviceToHost : cudaMemcpyHostToHost));
        if (h.magic != kCkMagic) fail("checkpoint: not a cavity checkpoint");
        if (h.nx != nx_ || h.ny != ny_ || h.nz != nz_ || h.field_bytes != (int)sizeof(T))
            fail("checkpoint: grid size or precision form differs from this solver");
        if (h.config_key != config_key())
            fail("checkpoint: saved by a solver with other settings (stretching, Re, lid, dt or solver options)");
        check(cudaMemcpyAsync(ctrl_, d + L.ctrl, sizeof(Control), kind, stream_));
        for (int k = 0; k < 3; k++) {
            check(cudaMemcpyAsync(U_[par_][k], d + L.u[k], sizeof(T) * size_[k], kind, stream_));
            check(cudaMemcpyAsync(M_[par_][k], d + L.m[k], sizeof(T) * size_[k], kind, stream_));
        }
        check(cudaMemcpyAsync(PHI_[par_], d + L.phi, sizeof(double) * n_cell_, kind, stream_));
        for (int k = 0; k < 4; k++) check(cudaMemcpyAsync(hist_[k], d + L.hist[k], sizeof(double) * n_cell_, kind, stream_));
        check(cudaMemcpyAsync(stats_, d + L.stats, sizeof(double) * 6 * nx_ * ny_, kind, stream_));
        check(cudaStreamSynchronize(stream_));
        pull_control();
        hc_.error = kOk;
        push_control();
        check(cudaStreamSynchronize(stream_));
    }
    void set_clock(double t, long long steps, double last_dt) override {
        hc_.t = t; hc_.steps = steps; hc_.last_dt = last_dt;
        push_control();
        check(cudaStreamSynchronize(stream_));
    }
    void probes(float* out) override {                                                // backend.cu:1159-1166
        if (c_.n_probes == 0) return;
        if (probes_fresh_) {           // the last step's tail computed them from the current state
            std::memcpy(out, tail_probes(), sizeof(float) * 2 * c_.n_probes);
            return;
        }
        probes_kernel<T><<<1, 32, 0, stream_>>>(out_args(), probe_cells_, c_.n_probes, probe_out_);
        check(cudaMemcpyAsync(out, probe_out_, sizeof(float) * 2 * c_.n_probes, cudaMemcpyDeviceToHost, stream_));
        check(cudaStreamSynchronize(stream_));
    }
    void add_statistics(double weight, double* centreline) override {                  // backend.cu:1168-1175
        statistics_kernel<T><<<blocks_for((long long)nx_ * ny_ + nx_), kThreads, 0, stream_>>>(out_args(), weight, nullptr, stats_, line_);
        check(cudaMemcpyAsync(centreline, line_, sizeof(double) * 5 * nx_, cudaMemcpyDeviceToHost, stream_));
        check(cudaStreamSynchronize(stream_));
    }
    void get_statistics(double* sums) override {
        check(cudaMemcpyAsync(sums, stats_, sizeof(double) * 6 * nx_ * ny_, cudaMemcpyDeviceToHost, stream_));
        check(cudaStreamSynchronize(stream_));
    }
    void set_statistics(const double* sums) override {
        check(cudaMemcpyAsync(stats_, sums, sizeof(double) * 6 * nx_ * ny_, cudaMemcpyHostToDevice, stream_));
        check(cudaStreamSynchronize(stream_));
    }
    void midplane(float* out) override {                                               // backend.cu:1178-1184
        midplane_kernel<T><<<blocks_for((long long)nx_ * ny_), kThreads, 0, stream_>>>(out_args(), (T)lid_speed_host(hc_.t), plane_);
        check(cudaMemcpyAsync(out, plane_, sizeof(float) * 4 * nx_ * ny_, cudaMemcpyDeviceToHost, stream_));
        check(cudaStreamSynchronize(stream_));
    }
    void q_volume(int colour_w, float* q, float* colour) override {                    // backend.cu:1185-1194
        const double L_over_U = c_.length / c_.u_lid;
        float* qd = fstage_;
        float* cd = fstage_ + n_cell_;
        q_kernel<T><<<blocks_for(n_cell_), kThreads, 0, stream_>>>(out_args(), (T)lid_speed_host(hc_.t), (T)(L_over_U * L_over_U),
                                                                  (T)(1.0 / c_.u_lid), colour_w, qd, cd);
        check(cudaMemcpyAsync(q, qd, sizeof(float) * n_cell_, cudaMemcpyDeviceToHost, stream_));
        check(cudaMemcpyAsync(colour, cd, sizeof(float) * n_cell_, cudaMemcpyDeviceToHost, stream_));
        check(cudaStreamSynchronize(stream_));
    }
    long long device_bytes() const override { return arena_.bytes(); }

    // step begin; per stage the sweep, the projection start, the residual of its guess and the finish; 7 per pass
    // step begin, then per stage the sweep, the projection start, its guess's residual and the finish, and per pass
    // the transforms' launches and the residual
    int kernels_per_step(int passes) const override { return 1 + 3 * 4 + 3 * passes * (transform_launches() + 1); }
    int transform_launches() const {
        if (tc_fdm_) return 6;
        const int f = pass_form(fdm_, form_env_ >= 0 ? form_env_ : tune_.fused);
        return f == kPassPairs ? 3 : f == kPassOneLaunch ? 1 : 6;
    }
    long long pressure_passes() const override { return hc_.pass_count; }

    // `steps` steps through the plain step graph, each timed by events around its launch; then, when `kms` is
    // given, `steps` more through the graph with events around the kernels (they cost launch latency, so the step
    // times come from the plain graph), for the per-kernel times
    void time_steps(int warmup, int steps, int flush, float* ms, float* kms) override {
        probes_fresh_ = false;
        if (flush && !flush_) check(cudaMalloc(&flush_, kFlushBytes));
        for (int i = 0; i < warmup; i++) step(nullptr);      // (the first may run the autotuner, which rebuilds graphs)
        ensure_graphs(false);
        if (kms) ensure_graphs(true);
        for (double& t : timed_ms_) t = 0;
        cudaEvent_t e0, e1;
        check(cudaEventCreate(&e0));
        check(cudaEventCreate(&e1));
        for (int pass = 0; pass < (kms ? 2 : 1); pass++) {
            const bool timing = pass == 1;
            for (int i = 0; i < steps; i++) {
                if (flush) check(cudaMemsetAsync(flush_, i & 0xff, kFlushBytes, stream_));
                check(cudaEventRecord(e0, stream_));
                if (eager_) enqueue_step(par_, timing, true);
                else check(cudaGraphLaunch(timing ? texec_[par_] : exec_[par_], stream_));
                pending_.push_back(par_);
                par_ ^= 1;
                check(cudaEventRecord(e1, stream_));
                sync(nullptr);
                if (!timing) {
                    check(cudaEventElapsedTime(&ms[i], e0, e1));
                    continue;
                }
                for (int kind = 0; kind < kNumTimed; kind++) {
                    float tot = 0, t;
                    for (int s = 0; s < 3; s++) {
                        check(cudaEventElapsedTime(&t, kev(kind, s)[0], kev(kind, s)[1]));
                        tot += t;
                    }
                    timed_ms_[kind] += tot / steps;
                    if (kind == kTkSweep) kms[i] = tot;
                }
            }
        }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
    }

    // Time whole steps under each candidate launch shape from the current state, restore the state after each,
    // and keep the fastest (cached per grid size, stretching and precision; see Tuning).  Two rounds: first the
    // momentum sweep (the tile kernel, in FP32 also its packed two-cells-per-thread form, or the march with 1/2, 1,
    // 2 and 4 times its device-filling z-chunk count;
    // only the chosen kernel when CAVITY_SWEEP names one), then, with the fastest sweep, the FP64 transforms where
    // they run (64 x 64 tiles, 32 x 32 tiles, 32 x 32 tiles in one cooperative launch, and three paired launches
    // where no axis exceeds 64 cells).
    void autotune(int steps, int* chunks_out, int* dgemm_out, int* fused_out, float* ms_out) override {
        if (!pending_.empty()) fail("autotune: steps are queued; sync first");
        steps = std::max(steps, 2);
        auto_tune_ = false;
        const long long bytes = checkpoint_bytes();
        void* saved = nullptr;
        check(cudaMalloc(&saved, (size_t)bytes));
        checkpoint_save(saved, 1);
        cudaEvent_t e0, e1;
        check(cudaEventCreate(&e0));
        check(cudaEventCreate(&e1));
        auto time_candidate = [&](const Tuning& cand) {
            tune_ = cand;
            if (cand.sweep >= 0) sweep_kind_ = cand.sweep;
            drop_graphs();
            float ms = -1;
            try {
                ensure_graphs(false);
                step(nullptr);                                   // warm-up (graph upload)
                check(cudaEventRecord(e0, stream_));
                for (int i = 0; i < steps; i++) {
                    check(cudaGraphLaunch(exec_[par_], stream_));
                    pending_.push_back(par_);
                    par_ ^= 1;
                }
                check(cudaEventRecord(e1, stream_));
                sync(nullptr);
                check(cudaEventElapsedTime(&ms, e0, e1));
                ms /= steps;
            } catch (const std::exception&) {
                ms = -1;                                         // a failed step: not a candidate
            }
            pending_.clear();
            checkpoint_load(saved, 1);
            return ms;
        };
        Tuning best;
        best.ms = -1;
        auto consider = [&](const Tuning& cand) {
            const float ms = time_candidate(cand);
            if (ms > 0 && (best.ms < 0 || ms < best.ms)) {
                best = cand;
                best.ms = ms;
            }
        };
        // round 1: the sweep
        const int forced = sweep_forced_ ? sweep_kind_ : -1;
        std::vector<Tuning> sweeps;
        if (forced < 0 || forced == kSweepTile) sweeps.push_back(Tuning{0, 0, -1, kSweepTile, 0});
        if (sizeof(T) == 4 && (forced < 0 || forced == kSweepPair)) sweeps.push_back(Tuning{0, 0, -1, kSweepPair, 0});
        if (forced < 0 || forced == kSweepMarch) {
            const int kind = sweep_kind_;
            sweep_kind_ = kSweepMarch;
            tune_ = Tuning{};
            const int c0 = (int)march_chunks();
            sweep_kind_ = kind;
            std::vector<int> cs;
            for (int c : {c0, c0 / 2, 2 * c0, 4 * c0}) {
                c = std::min(std::max(c, 1), std::max(1, nz_ / 4));
                if (std::find(cs.begin(), cs.end(), c) == cs.end()) cs.push_back(c);
            }
            for (int c : cs) sweeps.push_back(Tuning{c, 0, -1, kSweepMarch, 0});
        }
        if (forced == kSweepFace) sweeps.push_back(Tuning{0, 0, -1, kSweepFace, 0});
        for (const Tuning& t : sweeps) consider(t);
        // round 2: the FP64 transforms, with that sweep
        if (!tc_fdm_ && best.ms > 0) {
            std::vector<std::pair<int, int>> tiles = {{64, kPassSix}, {32, kPassSix}};
            if (fused_pass_capacity() > 0) tiles.push_back({32, kPassOneLaunch});
            if (pair_pass_fits(nx_, ny_, nz_)) tiles.push_back({0, kPassPairs});
            const Tuning sw = best;
            for (const auto& t : tiles) {
                Tuning cand = sw;
                cand.dgemm = t.first;
                cand.fused = t.second;
                consider(cand);
            }
        }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        cudaFree(saved);
        if (best.ms < 0) best = Tuning{};
        tune_ = best;
        if (best.sweep >= 0) sweep_kind_ = best.sweep;
        drop_graphs();
        if (best.ms > 0) tune_store(tune_key(c_, sizeof(T) == 8 ? 0 : 1), best);
        if (chunks_out) *chunks_out = best.chunks;
        if (dgemm_out) *dgemm_out = best.dgemm;
        if (fused_out) *fused_out = best.fused;
        if (ms_out) *ms_out = best.ms;
    }

    // per-step device time of the sweeps, the projection starts, the residuals of their guesses, the finishes and
    // the transforms of the first pass (all three stages) in the last time_steps call
    void kernel_times(double* ms) const override {
        for (int k = 0; k < kNumTimed; k++) ms[k] = timed_ms_[k];
    }

private:
    static constexpr size_t kFlushBytes = 256ull << 20;

    // ------------------------------------------------------------------------------ set-up
    void setup_params() {
        Params& p = p_;
        p.nx = nx_; p.ny = ny_; p.nz = nz_; p.n_cell = (int)n_cell_;
        p.o4 = c_.impulse_order == 4;
        p.adaptive_dt = c_.adaptive_dt; p.dt_lag = c_.dt_lag; p.phi_extrapolate = c_.phi_extrapolate;
        p.fdm_max_passes = c_.fdm_max_passes;
        p.nu = c_.nu; p.u_lid = c_.u_lid; p.lid_ramp_t = c_.lid_ramp_t; p.reinit_r = c_.reinit_r;
        p.dt_fixed = c_.dt_fixed; p.dt_max = c_.dt_max; p.cfl_target = c_.cfl_target;
        p.diffusion_limit = c_.diffusion_limit; p.fdm_rtol = c_.fdm_rtol;
        p.viscous_rate = (double)viscous_rate(c_, ax_);
        std::memset(&hc_, 0, sizeof hc_);
    }

    void allocate() {
        for (int s = 0; s < 3; s++) {
            for (int k = 0; k < 3; k++) {
                U_[s][k] = arena_.alloc<T>(size_[k]);
                M_[s][k] = arena_.alloc<T>(size_[k]);
            }
            PHI_[s] = arena_.alloc<double>(n_cell_);
        }
        for (int k = 0; k < 3; k++) M0_[k] = arena_.alloc<T>(size_[k]);
        phi0_ = arena_.alloc<double>(n_cell_);
        praw_ = arena_.alloc<double>(n_cell_);
        base_ = arena_.alloc<double>(n_cell_);
        rhs_ = arena_.alloc<double>(n_cell_);
        res_ = arena_.alloc<double>(n_cell_);
        for (int k = 0; k < 4; k++) hist_[k] = arena_.alloc<double>(n_cell_);
        t1_ = arena_.alloc<double>(n_cell_);
        t2_ = arena_.alloc<double>(n_cell_);
        inv_lambda_ = arena_.alloc<double>(n_cell_);
        // the grid-stride kernels' blocks, or the column kernels' plane blocks x z-chunks (at most one chunk per layer)
        partial_blocks_ = std::max((long long)blocks_for(std::max(max_face_, n_cell_)),
                                   (long long)blocks_for((long long)nx_ * ny_) * nz_) + 8;
        int sms = 148, dev = 0;
        check(cudaGetDevice(&dev));
        check(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        sms_ = sms;
        // the column kernels: how many of their blocks an SM holds (their grids fill the device that deep)
        check(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&start_per_sm_, (const void*)projection_start_kernel<T>,
                                                            kThreads, 0));
        check(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&residual_per_sm_, (const void*)residual_kernel, kThreads, 0));
        check(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&finish_per_sm_, (const void*)finish_kernel<T>, kThreads, 0));
        if (tc_fdm_) {
            inv_lambda_f_ = arena_.alloc<float>(n_cell_);
            const int n[3] = {nx_, ny_, nz_};
            for (int a = 0; a < 3; a++)
                for (int i = 0; i < 4; i++) img_[a][i] = arena_.alloc<float>(basis_image_floats(n[a], n[a]));
        }
        partial_ = arena_.alloc<double>(8 * partial_blocks_);
        ctrl_ = arena_.alloc<Control>(1);
        slots_ = arena_.alloc<double>(kNumSlots);
        out_counters_ = arena_.alloc<unsigned int>(kNumOutCounters);
        stats_ = arena_.alloc<double>(6LL * nx_ * ny_);
        line_ = arena_.alloc<double>(5LL * nx_);
        plane_ = arena_.alloc<float>(4LL * nx_ * ny_);
        fstage_ = arena_.alloc<float>(std::max(max_face_, 2 * n_cell_));
        dstage_[0] = arena_.alloc<double>(max_face_);
        dstage_[1] = arena_.alloc<double>(max_face_);
        probe_cells_ = arena_.alloc<int>(24);
        probe_out_ = arena_.alloc<float>(16);
    }

    void upload_tables() {
        Geo<T>& g = geo_;
        for (int a = 0; a < 3; a++) {
            const AxisGrid& ag = ax_[a];
            const int stride = tab_stride(ag.n);
            const std::vector<T> t = axis_tables<T>(ag, c_.impulse_order4_ramp, stride);
            T* d = arena_.alloc<T>((long long)t.size());
            check(cudaMemcpy(d, t.data(), sizeof(T) * t.size(), cudaMemcpyHostToDevice));
            g.tab[a] = d;
            g.stride[a] = stride;
            std::vector<double> inv(ag.n + 1);
            for (int i = 0; i <= ag.n; i++) inv[i] = 1.0 / ag.spacing[i];
            double* dw = arena_.alloc<double>(ag.n);
            double* di = arena_.alloc<double>(ag.n + 1);
            check(cudaMemcpy(dw, ag.width.data(), sizeof(double) * ag.n, cudaMemcpyHostToDevice));
            check(cudaMemcpy(di, inv.data(), sizeof(double) * (ag.n + 1), cudaMemcpyHostToDevice));
            g.dw[a] = dw;
            g.dinv_sp[a] = di;
            double* cen = arena_.alloc<double>(ag.n);
            check(cudaMemcpy(cen, ag.centre.data(), sizeof(double) * ag.n, cudaMemcpyHostToDevice));
            centre_[a] = cen;
        }
        const std::vector<T> lid = lid_u_table<T>(c_, ax_);
        T* dl = arena_.alloc<T>((long long)lid.size());
        check(cudaMemcpy(dl, lid.data(), sizeof(T) * lid.size(), cudaMemcpyHostToDevice));
        g.lid_u = dl;
        // pressure eigenbases (FP64) and 1/(lambda_x + lambda_y + lambda_z), 0 at the constant mode
        AxisEigen e[3];
        for (int a = 0; a < 3; a++) {
            e[a] = axis_eigen_shared(ax_[a]);
            const int n = ax_[a].n;
            std::vector<double> st((size_t)n * n);
            for (int i = 0; i < n; i++)
                for (int j = 0; j < n; j++) st[(size_t)j * n + i] = e[a].S[(size_t)i * n + j];
            S_[a] = arena_.alloc<double>((long long)n * n);
            ST_[a] = arena_.alloc<double>((long long)n * n);
            check(cudaMemcpy(S_[a], e[a].S.data(), sizeof(double) * n * n, cudaMemcpyHostToDevice));
            check(cudaMemcpy(ST_[a], st.data(), sizeof(double) * n * n, cudaMemcpyHostToDevice));
        }
        std::vector<double> inv((size_t)n_cell_);
        for (int z = 0; z < nz_; z++)
            for (int y = 0; y < ny_; y++)
                for (int x = 0; x < nx_; x++) {
                    const bool zero = x == e[0].zero_mode && y == e[1].zero_mode && z == e[2].zero_mode;
                    inv[x + (size_t)nx_ * (y + (size_t)ny_ * z)] =
                        zero ? 0.0 : 1.0 / (e[2].lambda[z] + e[1].lambda[y] + e[0].lambda[x]);
                }
        check(cudaMemcpy(inv_lambda_, inv.data(), sizeof(double) * n_cell_, cudaMemcpyHostToDevice));
        // The arena's zero-fills and these uploads run on the legacy default stream, and a copy from pageable
        // memory may return before its DMA has landed; stream_ is non-blocking, so wait for that stream before
        // kernels on stream_ read the uploaded operators (only for it: other solvers' streams keep running).
        check(cudaStreamSynchronize(cudaStreamLegacy));
        if (tc_fdm_) {
            // float S and 1/lambda as the reference keeps them (backend.cu:766-786), S split into hi/lo TF32
            // images of its rows (img 0, 1) and of its columns = rows of S^T (img 2, 3)
            convert_kernel<double, float><<<blocks_for(n_cell_), kThreads, 0, stream_>>>(inv_lambda_, inv_lambda_f_,
                                                                                          n_cell_);
            tcop_.nx = nx_; tcop_.ny = ny_; tcop_.nz = nz_;
            tcop_.inv_lambda = inv_lambda_f_;
            for (int a = 0; a < 3; a++) {
                launch_basis_image(stream_, S_[a], ax_[a].n, 0, img_[a][0], img_[a][1]);
                launch_basis_image(stream_, S_[a], ax_[a].n, 1, img_[a][2], img_[a][3]);
                for (int i = 0; i < 4; i++) tcop_.img[a][i] = img_[a][i];
            }
            check(cudaGetLastError());
        }
        fdm_.nx = nx_; fdm_.ny = ny_; fdm_.nz = nz_;
        for (int a = 0; a < 3; a++) { fdm_.s[a] = S_[a]; fdm_.st[a] = ST_[a]; }
        fdm_.inv_lambda = inv_lambda_;
        const std::vector<int> cells = probe_cells(c_, ax_);
        if (!cells.empty()) check(cudaMemcpy(probe_cells_, cells.data(), sizeof(int) * cells.size(), cudaMemcpyHostToDevice));
        check(cudaStreamSynchronize(cudaStreamLegacy));
        push_control();
    }

    double lid_speed_host(double time) const {
        if (c_.lid_ramp_t > 0) return c_.u_lid * std::min(1.0, std::max(time, 0.0) / c_.lid_ramp_t);
        return c_.u_lid;
    }

    void push_control() {
        hc_.counter[kCntBar] = 0;         // a grid barrier that timed out may have left arrivals behind
        check(cudaMemcpyAsync(ctrl_, &hc_, sizeof hc_, cudaMemcpyHostToDevice, stream_));
    }
    void pull_control() {
        check(cudaMemcpyAsync(&hc_, ctrl_, sizeof hc_, cudaMemcpyDeviceToHost, stream_));
        check(cudaStreamSynchronize(stream_));
    }

    [[noreturn]] void raise_error(int code) {
        char msg[200];
        switch (code) {
        case kVelocityNaN: fail("velocity is NaN/inf: the solution has blown up");
        case kRhsNaN: fail("pressure solve: right-hand side is NaN/inf (the run has blown up)");
        case kResidualNaN: fail("pressure solve: residual is NaN/inf");
        case kDeviceWait: fail("pressure solve: a tensor-core transform timed out waiting for its MMAs");
        case kBarrierWait: fail("pressure solve: the one-launch FDM pass timed out at a grid barrier");
        case kNotConverged:
            std::snprintf(msg, sizeof msg, "pressure solve: residual %.2e > FDM_RTOL after %d passes", hc_.error_value,
                          hc_.error_passes);
            fail(msg);
        default: fail("solver error " + std::to_string(code));
        }
    }

    OutArgs<T> out_args() const {
        OutArgs<T> a;
        a.p = p_;
        a.g = geo_;
        for (int k = 0; k < 3; k++) { a.u[k] = U_[par_][k]; a.m[k] = M_[par_][k]; }
        a.centre_x = centre_[0];
        a.centre_z = centre_[2];
        a.length_x = (double)(float)ax_[0].length;
        a.length_z = (double)(float)ax_[2].length;
        a.lid_shaped = c_.lid_shaped;
        a.slots = slots_;
        a.partial = partial_;
        a.counters = out_counters_;
        return a;
    }

    void update_cfl() {
        CflArgs<T> a;
        a.p = p_;
        a.g = geo_;
        for (int k = 0; k < 3; k++) a.u[k] = U_[par_][k];
        a.c = ctrl_;
        a.partial = partial_;
        cfl_kernel<T><<<blocks_for(n_cell_), kThreads, 0, stream_>>>(a);
    }

    // ------------------------------------------------------------------------------ kernel launches
    // grid of a column kernel (ColumnSpan): plane blocks along x and z-chunks along y, as many chunks as it takes
    // for the launch (all cavities of a batch together) to fill the device `per_sm` blocks deep in one wave, or
    // about four waves when the plane blocks alone exceed one
    dim3 column_grid(int per_sm, int per_thread = 1) const {
        const long long bpp = blocks_for((long long)nx_ * ny_ / per_thread);
        const long long want = (long long)sms_ * std::max(per_sm, 1);
        const long long cav = std::max(g_launch_batch, 1);
        long long chunks = want / (bpp * cav);
        // a launch that holds more plane blocks than fit at once (a large batch): chunks for about four waves, so
        // that the last, partial wave is a small share of the launch
        if (chunks < 1) chunks = (4 * want + bpp * cav - 1) / (bpp * cav);
        chunks = std::min<long long>(nz_, std::max(1LL, chunks));
        const long long zc = (nz_ + chunks - 1) / chunks;
        chunks = (nz_ + zc - 1) / zc;
        return dim3((unsigned int)bpp, (unsigned int)chunks);
    }
    void launch_step_begin(cudaStream_t st) {
        StepBeginArgs a;
        a.p = p_;
        a.c = ctrl_;
        if (!record_launch(kLkStepBegin, 0, dim3(1), 0, a)) check(launch_pdl(step_begin_kernel, dim3(1), dim3(32), 0, st, p_, ctrl_));
    }
    void launch_momentum(cudaStream_t st, int stage, int S, int in, int out) {
        MomentumArgs<T> a;
        a.p = p_;
        a.g = geo_;
        for (int k = 0; k < 3; k++) {
            a.u[k] = U_[in][k];
            a.m[k] = M_[stage == 0 ? S : in][k];
            a.m0[k] = M0_[k];
            a.m0_out[k] = M0_[k];
            a.out[k] = M_[out][k];
        }
        a.c = ctrl_;
        a.stage = stage;
        a.r = (T)c_.reinit_r;
        a.one_minus_r = (T)(1.0 - c_.reinit_r);
        a.nu = (T)c_.nu;
        if (sweep_kind_ == kSweepMarch) {
            using G = MarchG;
            const dim3 grid((nx_ + G::TX - 1) / G::TX, (ny_ + G::TY - 1) / G::TY, march_chunks());
            if (!record_launch(kLkSweep, kSweepMarch, grid, G::template smem_bytes<T>(), a))
                check(launch_pdl(sweep_march_kernel<T, kMarchTX, kMarchTY>, grid, dim3(G::NT),
                                 G::template smem_bytes<T>(), st, a));
        } else if (sweep_kind_ == kSweepPair) {
            if constexpr (sizeof(T) == 4) {
                const dim3 grid((nx_ + TileG::TX - 1) / TileG::TX, (ny_ + kTileTY - 1) / kTileTY, (nz_ + kTileTZ - 1) / kTileTZ);
                const size_t smem = PairG::template smem_bytes<T>();
                if (!record_launch(kLkSweep, kSweepPair, grid, smem, a))
                    check(launch_pdl(sweep_pair_kernel<kTileTY, kTileTZ, kPairNT>, grid, dim3(kPairNT), smem, st, a));
            } else {
                fail("the packed sweep is FP32 only");
            }
        } else if (sweep_kind_ == kSweepTile) {
            using G = TileG;
            dim3 grid((nx_ + G::TX - 1) / G::TX, (ny_ + kTileTY - 1) / kTileTY, (nz_ + kTileTZ - 1) / kTileTZ);
            if (!record_launch(kLkSweep, kSweepTile, grid, G::template smem_bytes<T>(), a))
                check(launch_pdl(sweep_tile_kernel<T, kTileTY, kTileTZ, kTileNT>, grid, dim3(kTileNT),
                                 G::template smem_bytes<T>(), st, a));
        } else {
            dim3 grid(blocks_for(max_face_), 3);
            momentum_kernel<T><<<grid, kThreads, 0, st>>>(a);
        }
    }
    // rhs, starting potential and its residual, start-of-solve decisions (backend.cu:816-831)
    // use_h: 0 no graph loop, 1 this solver's own loop, 2 a loop shared by a batch (see set_loop); `between` runs
    // between the start kernel and the residual of the guess (timing events)
    void launch_start(cudaStream_t st, T* const m[3], bool step_mode, int stage, int S, int cur,
                      cudaGraphConditionalHandle h, int use_h, const std::function<void()>& between = {}) {
        StartArgs<T> a;
        a.p = p_;
        a.g = geo_;
        for (int k = 0; k < 3; k++) a.m[k] = m[k];
        a.rhs = rhs_;
        a.res = res_;
        a.guess = praw_;
        a.phi_state = PHI_[S];
        a.phi0 = phi0_;
        a.phi_cur = PHI_[cur];
        a.base = step_mode ? base_ : nullptr;
        for (int k = 0; k < 4; k++) a.hist[k] = hist_[k];
        a.stage = stage;
        a.c = ctrl_;
        a.partial = partial_;
        a.handle = h;
        a.use_handle = use_h;
        const dim3 grid = column_grid(start_per_sm_);
        if (!record_launch(kLkStart, 0, grid, 0, a))
            check(launch_pdl(projection_start_kernel<T>, grid, dim3(kThreads), 0, st, a));
        if (between) between();
        if (step_mode) launch_residual(st, praw_, h, use_h, 1);    // the residual of the guess
    }
    void launch_residual(cudaStream_t st, const double* phi, cudaGraphConditionalHandle h, int use_h, int start = 0) {
        ResidualArgs a;
        a.start = start;
        a.p = p_;
        for (int k = 0; k < 3; k++) { a.dw[k] = geo_.dw[k]; a.dinv_sp[k] = geo_.dinv_sp[k]; }
        a.phi = phi;
        a.rhs = rhs_;
        a.res = res_;
        a.c = ctrl_;
        a.partial = partial_;
        a.handle = h;
        a.use_handle = use_h;
        const dim3 grid = column_grid(residual_per_sm_, 2);     // a pair of cells per thread
        if (!record_launch(kLkResidual, 0, grid, 0, a)) check(launch_pdl(residual_kernel, grid, dim3(kThreads), 0, st, a));
    }
    // one pressure pass (backend.cu:801-814) followed by the residual that decides on the next
    void launch_pass(cudaStream_t st, double* phi, cudaGraphConditionalHandle h, int use_h) {
        launch_transforms(st, phi, h, use_h);
        launch_residual(st, phi, h, use_h);
    }
    // the six transforms of a pass (backend.cu:801-814)
    void launch_transforms(cudaStream_t st, double* phi, cudaGraphConditionalHandle h, int use_h) {
        if (tc_fdm_) launch_tc_pass(st, phi, h, use_h != 0);
        else {
            const int outer = g_dgemm_tile;              // a batch's choice wins over this cavity's own tuning
            if (!g_launch_record && tune_.dgemm) g_dgemm_tile = tune_.dgemm;
            launch_fdm_pass(st, fdm_, res_, rhs_, phi, t1_, t2_, ctrl_, h, use_h != 0,
                            form_env_ >= 0 ? form_env_ : tune_.fused);
            g_dgemm_tile = outer;
        }
    }
    void launch_tc_pass(cudaStream_t st, double* phi, cudaGraphConditionalHandle h, bool use_h) {
        launch_tc_fdm_pass(st, tcop_, res_, rhs_, phi, reinterpret_cast<float*>(t1_), reinterpret_cast<float*>(t2_),
                           ctrl_, h, use_h, sms_);
    }
    void launch_finish(cudaStream_t st, T* const m[3], T* const u_out[3], double* phi_out, bool step_mode, int stage,
                       bool last) {
        FinishArgs<T> a;
        a.p = p_;
        a.g = geo_;
        for (int k = 0; k < 3; k++) { a.m[k] = m[k]; a.u_out[k] = u_out[k]; }
        a.phi = praw_;
        a.phi_out = phi_out;
        a.base = base_;
        for (int k = 0; k < 4; k++) a.hist[k] = hist_[k];
        a.step_mode = step_mode;
        a.last_stage = last;
        a.stage = stage;
        a.c = ctrl_;
        a.partial = partial_;
        const dim3 grid = column_grid(finish_per_sm_);
        if (!record_launch(kLkFinish, 0, grid, 0, a)) check(launch_pdl(finish_kernel<T>, grid, dim3(kThreads), 0, st, a));
    }

    // A pressure refinement loop inside a stream capture: one pass, then a conditional while-node whose body is
    // one pass.  `first_residual` launches the kernels that set the loop condition before them.
    template <class F>
    void captured_loop(F first_residual, double* phi, cudaEvent_t t0 = nullptr, cudaEvent_t t1 = nullptr) {
        cudaStreamCaptureStatus status;
        cudaGraph_t g;
        const cudaGraphNode_t* deps;
        size_t ndeps;
        check(cudaStreamGetCaptureInfo(stream_, &status, nullptr, &g, &deps, &ndeps));
        cudaGraphConditionalHandle h;
        check(cudaGraphConditionalHandleCreate(&h, g, 0, cudaGraphCondAssignDefault));
        first_residual(h);
        // the first pass outside the loop: most solves need exactly one, and its kernels skip themselves when the
        // start decided on none (the first transform clears the loop condition either way)
        if (t0) check(cudaEventRecordWithFlags(t0, stream_, cudaEventRecordExternal));
        launch_transforms(stream_, phi, h, 1);
        if (t1) check(cudaEventRecordWithFlags(t1, stream_, cudaEventRecordExternal));
        launch_residual(stream_, phi, h, 1);
        check(cudaStreamGetCaptureInfo(stream_, &status, nullptr, &g, &deps, &ndeps));
        cudaGraphNodeParams cp = {cudaGraphNodeTypeConditional};
        cp.type = cudaGraphNodeTypeConditional;
        cp.conditional.handle = h;
        cp.conditional.type = cudaGraphCondTypeWhile;
        cp.conditional.size = 1;
        cudaGraphNode_t node;
        check(cudaGraphAddNode(&node, g, deps, ndeps, &cp));
        cudaGraph_t body = cp.conditional.phGraph_out[0];
        check(cudaStreamBeginCaptureToGraph(body_stream_, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed));
        launch_pass(body_stream_, phi, h, 1);
        check(cudaStreamEndCapture(body_stream_, &body));
        check(cudaStreamUpdateCaptureDependencies(stream_, &node, 1, cudaStreamSetCaptureDependencies));
    }

    // The time step for state parity S (backend.cu:877-955), enqueued on stream_: under stream capture (the
    // refinement loops become conditional while-nodes), or eagerly with the loops driven from the host (the
    // launch mode for profilers, which cannot see kernels inside graphs that hold conditional nodes).
    void enqueue_step(int S, bool timing, bool eager) {
        const int Xs = S ^ 1, Ys = 2;
        auto mark = [&](cudaEvent_t e) {
            if (eager) check(cudaEventRecord(e, stream_));
            else check(cudaEventRecordWithFlags(e, stream_, cudaEventRecordExternal));
        };
        launch_step_begin(stream_);
        for (int stage = 0; stage < 3; stage++) {
            const int in = stage == 0 ? S : stage == 1 ? Xs : Ys;
            const int out = stage == 1 ? Ys : Xs;
            const int cur = stage == 1 ? Xs : Ys;          // potential of the previous stage (stages 1, 2)
            if (timing) mark(kev(kTkSweep, stage)[0]);
            launch_momentum(stream_, stage, S, in, out);
            if (timing) mark(kev(kTkSweep, stage)[1]);
            double* phi = praw_;          // the solve works here; finish writes PHI_[out]
            // with timing: events around the projection start and around the residual of its guess
            std::function<void()> between;
            if (timing) {
                mark(kev(kTkStart, stage)[0]);
                between = [&, stage] {
                    mark(kev(kTkStart, stage)[1]);
                    mark(kev(kTkGuessResidual, stage)[0]);
                };
            }
            if (eager) {
                launch_start(stream_, M_[out], true, stage, S, cur, 0, 0, between);
                if (timing) mark(kev(kTkGuessResidual, stage)[1]);
                pull_control();
                for (int pass = 0; hc_.cond && !hc_.error; pass++) {
                    if (timing && pass == 0) mark(kev(kTkTransforms, stage)[0]);
                    launch_transforms(stream_, phi, 0, 0);
                    if (timing && pass == 0) mark(kev(kTkTransforms, stage)[1]);
                    launch_residual(stream_, phi, 0, 0);
                    pull_control();
                }
            } else {
                captured_loop([&](cudaGraphConditionalHandle h) {
                    launch_start(stream_, M_[out], true, stage, S, cur, h, 1, between);
                    if (timing) mark(kev(kTkGuessResidual, stage)[1]);
                }, phi, timing ? kev(kTkTransforms, stage)[0] : nullptr, timing ? kev(kTkTransforms, stage)[1] : nullptr);
            }
            if (timing) mark(kev(kTkFinish, stage)[0]);
            launch_finish(stream_, M_[out], U_[out], PHI_[out], true, stage, stage == 2);
            if (timing) mark(kev(kTkFinish, stage)[1]);
        }
    }

    void build_graphs() {
        {
            // momentum sweep: shared-memory tiles (FP32: two cells per thread, packed) unless CAVITY_SWEEP=march (the
            // z-march, sweep_march.cuh), =face (a thread per face) or =tile (one cell per thread).  The march evaluates each edge once but measured slower than the tiles (C2:
            // 54.6 against 40.6 us per launch; 128^3 mixed: 196 against 133 us), so it is not the default.
            const char* sw = std::getenv("CAVITY_SWEEP");
            const std::string kind = sw ? sw : "";
            sweep_kind_ = kind == "face" ? kSweepFace : kind == "march" ? kSweepMarch : kSweepTile;
            // the FP32 default is the packed two-cells-per-thread tile kernel (sweep_pair.cuh); CAVITY_SWEEP=tile
            // selects one cell per thread
            if (kind == "pair" || (kind.empty() && sizeof(T) == 4)) sweep_kind_ = sizeof(T) == 4 ? kSweepPair : kSweepTile;
            sweep_forced_ = !kind.empty();
            check(cudaFuncSetAttribute(sweep_tile_kernel<T, kTileTY, kTileTZ, kTileNT>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TileG::template smem_bytes<T>()));
            if constexpr (sizeof(T) == 4)
                check(cudaFuncSetAttribute(sweep_pair_kernel<kTileTY, kTileTZ, kPairNT>,
                                           cudaFuncAttributeMaxDynamicSharedMemorySize, (int)PairG::template smem_bytes<T>()));
            {
                const int smem = (int)MarchG::template smem_bytes<T>();
                check(cudaFuncSetAttribute(sweep_march_kernel<T, kMarchTX, kMarchTY>,
                                           cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
                check(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&march_per_sm_, sweep_march_kernel<T, kMarchTX, kMarchTY>,
                                                                    MarchG::NT, smem));
                march_per_sm_ = std::max(1, march_per_sm_);
            }
            if (tc_fdm_) check(tc_transform_prepare());
            check(pair_prepare());
            form_env_ = pass_form_from_env();
        }
        for (cudaEvent_t& e : kev_) check(cudaEventCreate(&e));
        const char* env = std::getenv("CAVITY_GRAPHS");
        eager_ = env && env[0] == '0';
    }
    // the step graphs of both state parities (timing: with events around the sweeps), captured on first use, so
    // a solver that only takes part in batches or is only initialised never builds them
    void drop_graphs() {
        for (int s = 0; s < 2; s++) {
            if (exec_[s]) cudaGraphExecDestroy(exec_[s]);
            if (graph_[s]) cudaGraphDestroy(graph_[s]);
            if (texec_[s]) cudaGraphExecDestroy(texec_[s]);
            if (tgraph_[s]) cudaGraphDestroy(tgraph_[s]);
            exec_[s] = texec_[s] = nullptr;
            graph_[s] = tgraph_[s] = nullptr;
        }
    }
    void ensure_graphs(bool timing) {
        if (eager_) return;
        for (int S = 0; S < 2; S++) {
            cudaGraph_t& g = timing ? tgraph_[S] : graph_[S];
            cudaGraphExec_t& ex = timing ? texec_[S] : exec_[S];
            if (ex) continue;
            check(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal));
            enqueue_step(S, timing, false);
            check(cudaStreamEndCapture(stream_, &g));
            check(cudaGraphInstantiate(&ex, g, 0));
        }
    }

    // A projection outside a step (initialize, kick): m -> u, phi from no guess (backend.cu:849-854), with
    // the refinement loop driven from the host.  Also refreshes the CFL rate of u.
    void project(T* const m[3], double* phi, T* const u_out[3]) {
        hc_.error = kOk;
        push_control();
        for (int k = 0; k < 3; k++) zero_walls_kernel<T><<<blocks_for(size_[k]), kThreads, 0, stream_>>>(p_, k, m[k]);
        launch_start(stream_, m, false, 0, par_, par_, 0, 0);
        pull_control();
        int guard = 0;
        while (hc_.cond && !hc_.error && guard++ < 1000) {
            launch_pass(stream_, praw_, 0, 0);
            pull_control();
        }
        if (hc_.error) {
            const int code = hc_.error;
            hc_.error = kOk;
            push_control();
            check(cudaStreamSynchronize(stream_));
            raise_error(code);
        }
        launch_finish(stream_, m, u_out, phi, false, 0, true);
        pull_control();
    }

    CavityConfig c_;
    int nx_, ny_, nz_;
    long long n_cell_, size_[3], max_face_;
    AxisGrid ax_[3];
    double volume_;
    Params p_;
    Geo<T> geo_;
    Control hc_;
    DeviceArena arena_;
    cudaStream_t stream_ = nullptr, body_stream_ = nullptr;
    int par_ = 0;
    bool eager_ = false;
    int sweep_kind_ = kSweepTile;
    bool sweep_forced_ = false;         // CAVITY_SWEEP named the kernel
    Tuning tune_;
    bool auto_tune_ = false;
    int form_env_ = -1;                 // FP64 pass form named by CAVITY_FDM_FUSED at creation (-1: none)
    int march_per_sm_ = 1;
    // z-chunks of a march sweep launch: as many as fill the device's resident CTA slots once (all cavities of a
    // batch together) with at least four layers per chunk; CAVITY_MARCH_CHUNKS overrides
    unsigned int march_chunks() const {
        const long long tiles = (long long)((nx_ + kMarchTX - 1) / kMarchTX) * ((ny_ + kMarchTY - 1) / kMarchTY) *
                                std::max(g_launch_batch, 1);
        long long chunks = (long long)sms_ * march_per_sm_ / tiles;
        if (tune_.chunks > 0 && g_launch_batch <= 1) chunks = tune_.chunks;
        if (const char* e = std::getenv("CAVITY_MARCH_CHUNKS")) chunks = std::atoll(e);
        chunks = std::min<long long>(std::max(1LL, chunks), std::max(1, nz_ / 4));
        const long long zc = (nz_ + chunks - 1) / chunks;
        return (unsigned int)((nz_ + zc - 1) / zc);
    }
    std::vector<int> pending_;
    long long steps_before_ = 0;
    // fields: three buffer sets of velocity, impulse and potential (state, stage outputs)
    T* U_[3][3];
    T* M_[3][3];
    double* PHI_[3];
    T* M0_[3];
    double *phi0_, *praw_, *base_, *rhs_, *res_, *hist_[4], *t1_, *t2_, *inv_lambda_;
    double *S_[3], *ST_[3];
    FdmOperands fdm_;
    bool tc_fdm_ = false;              // mixed form: tcgen05 transforms
    int sms_ = 148;
    float* inv_lambda_f_ = nullptr;
    float* img_[3][4] = {};            // per axis: S rows hi, lo; S^T rows hi, lo (basis images)
    TcFdmOperands tcop_ = {};
    double* partial_;
    long long partial_blocks_;
    int residual_per_sm_ = 1, start_per_sm_ = 1, finish_per_sm_ = 1;
    Control* ctrl_;
    double *slots_, *stats_, *line_, *dstage_[2];
    unsigned int* out_counters_;
    float *plane_, *fstage_, *probe_out_;
    int* probe_cells_;
    const double* centre_[3];
    cudaGraph_t graph_[2] = {nullptr, nullptr}, tgraph_[2] = {nullptr, nullptr};
    cudaGraphExec_t exec_[2] = {nullptr, nullptr}, texec_[2] = {nullptr, nullptr};
    // events of the timing graph: [kernel][stage][begin, end]; per-step means of the last time_steps call
    enum TimedKernel : int { kTkSweep = 0, kTkStart, kTkGuessResidual, kTkFinish, kTkTransforms, kNumTimed };
    cudaEvent_t kev_[2 * 3 * kNumTimed] = {};
    cudaEvent_t* kev(int kind, int stage) { return kev_ + 2 * (3 * kind + stage); }
    double timed_ms_[kNumTimed] = {};
    void* flush_ = nullptr;
    // the step tail's outputs (step_tail_kernel): one pinned, mapped block holding the control block and the probe
    // values after the last step queued through step_async
    void* tail_host_ = nullptr;
    void* tail_dev_ = nullptr;
    bool tail_queued_ = false;          // the last queued step has its tail
    bool probes_fresh_ = false;         // the tail's probe values are those of the current state
    Control* tail_control() const { return static_cast<Control*>(tail_host_); }
    float* tail_probes() const { return reinterpret_cast<float*>(static_cast<char*>(tail_host_) + 256 * ((sizeof(Control) + 255) / 256)); }
    float* ring_host_ = nullptr;       // queued per-step probe values (pinned, mapped)
    float* ring_dev_ = nullptr;
    int ring_n_ = 0;
};


// ------------------------------------------------------------------------------------------------ batches
// B cavities of the same grid size and form stepped together by one CUDA graph per state parity, each of whose
// kernel launches covers every cavity (the batched entries of the kernels: grid axis z runs over the cavities,
// and each block reads its cavity's argument record from a device array).  The launch sequence and the
// argument records are the members' own: each member's launch helpers run with a recorder installed.  The
// refinement loop of a stage runs while any cavity needs another pass; a cavity whose solve has ended skips
// the later passes.  Every cavity keeps its own control block, dt, pass count, clock and errors, and stays a
// full solver between steps (getters, kick, fields through its own handle).
class BatchBase {
public:
    virtual ~BatchBase() {}
    virtual void step_async(int count) = 0;
    virtual void sync(CavityReport* reports) = 0;
    virtual int size() const = 0;
    virtual void set_member(int slot, SolverBase* s) = 0;
    virtual void part_times(int steps, double* ms) = 0;
};

template <class T> class Batch : public BatchBase {
    using S_ = Solver<T>;
    static constexpr int kTY = S_::kTileTY, kTZ = S_::kTileTZ, kNT = S_::kTileNT;

public:
    // `members` fill slots 0 .. n-1 of `capacity` slots; the other slots start empty (cavities of one size only)
    Batch(const std::vector<S_*>& members, int capacity) : m_(members) {
        if (m_.empty()) fail("batch: no cavities");
        const S_& f = *m_[0];
        long long tiles64 = 0;
        for (const S_* s : m_) {
            if (s->nx_ != f.nx_ || s->ny_ != f.ny_ || s->nz_ != f.nz_) mixed_sizes_ = true;
            tiles64 += (long long)((s->nx_ + 63) / 64) * ((s->ny_ * s->nz_ + 63) / 64);
            check_member(s, f);
        }
        for (size_t i = 0; i < m_.size(); i++)
            for (size_t k = 0; k < i; k++)
                if (m_[i] == m_[k]) fail("batch: a cavity appears twice");
        if (capacity < (int)m_.size()) capacity = (int)m_.size();
        if (capacity > (int)m_.size() && mixed_sizes_) fail("batch: empty slots need cavities of one grid size");
        // cavities of different sizes share one FP64 transform tile: the large one when all of them together
        // have two 64 x 64 tiles per SM in the largest transform
        if (mixed_sizes_) dgemm_tile_ = tiles64 >= 2 * f.sms_ ? 64 : 32;
        // FP64 passes as paired launches when every member's axes allow them (and CAVITY_FDM_FUSED names no
        // other form)
        {
            bool fits = true;
            for (const S_* s : m_) fits = fits && pair_pass_fits(s->nx_, s->ny_, s->nz_);
            const int e = pass_form_from_env();
            pairs_ = fits && (e < 0 || e == kPassPairs) ? 1 : 0;
        }
        proto_ = m_[0];
        par_ = m_[0]->par_;
        nx_ = f.nx_;
        ny_ = f.ny_;
        nz_ = f.nz_;
        tc_fdm_ = f.tc_fdm_;
        sweep_kind_ = f.sweep_kind_;
        m_.resize(capacity, nullptr);
        d_.assign(capacity, 0);
        for (int i = 0; i < capacity; i++)
            if (m_[i]) d_[i] = m_[i]->par_ ^ par_;
        check(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
        check(cudaStreamCreateWithFlags(&body_stream_, cudaStreamNonBlocking));
        using G = TileGeom<kTY, kTZ, kNT>;
        check(cudaFuncSetAttribute(sweep_tile_batched<T, kTY, kTZ, kNT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)G::template smem_bytes<T>()));
        check(cudaFuncSetAttribute(sweep_march_batched<T, S_::kMarchTX, S_::kMarchTY>,
                                   cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)S_::MarchG::template smem_bytes<T>()));
        if constexpr (sizeof(T) == 4)
            check(cudaFuncSetAttribute(sweep_pair_batched<kTY, kTZ, S_::kPairNT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)S_::PairG::template smem_bytes<T>()));
        if (f.tc_fdm_) check(tc_transform_prepare_batched());
        check(pair_prepare());
        for (int S = 0; S < 2; S++) build(S);
        proto_ = nullptr;        // members may leave and be destroyed from now on
    }
    ~Batch() override {
        if (stream_) cudaStreamSynchronize(stream_);
        for (int S = 0; S < 2; S++) {
            if (exec_[S]) cudaGraphExecDestroy(exec_[S]);
            if (graph_[S]) cudaGraphDestroy(graph_[S]);
            if (dargs_[S]) cudaFree(dargs_[S]);
        }
        drop_timing();
        for (cudaEvent_t& e : tev_)
            if (e) cudaEventDestroy(e);
        if (stream_) cudaStreamDestroy(stream_);
        if (body_stream_) cudaStreamDestroy(body_stream_);
    }
    int size() const override { return (int)m_.size(); }

    void step_async(int count) override {
        for (int i = 0; i < count; i++) launch_step(exec_);
    }
    // Per-step device time (ms, summed over the three stages) of the batch's parts: the sweeps, the projection
    // starts with the residuals of their guesses, the first pressure pass of each stage (transforms and
    // residual), and the finishes, over `steps` steps through a second graph with events between the parts.
    // The steps advance the cavities as cavity_batch_step_async does (the same kernels in the same order).
    void part_times(int steps, double* ms) override {
        if (queued_) fail("batch: steps are queued; sync first");
        if (!tev_[0])
            for (cudaEvent_t& e : tev_) check(cudaEventCreate(&e));
        drop_timing();
        for (int S = 0; S < 2; S++) build(S, true);
        for (int k = 0; k < kParts; k++) ms[k] = 0;
        for (int i = 0; i < steps; i++) {
            launch_step(texec_);
            sync(nullptr);
            for (int stage = 0; stage < 3; stage++)
                for (int k = 0; k < kParts; k++) {
                    float t = 0;
                    check(cudaEventElapsedTime(&t, tev_[(stage * kParts + k) * 2], tev_[(stage * kParts + k) * 2 + 1]));
                    ms[k] += t / std::max(steps, 1);
                }
        }
    }
    static constexpr int kParts = 4;

private:
    void drop_timing() {
        for (int S = 0; S < 2; S++) {
            if (texec_[S]) cudaGraphExecDestroy(texec_[S]);
            if (tgraph_[S]) cudaGraphDestroy(tgraph_[S]);
            if (targs_[S]) cudaFree(targs_[S]);
            texec_[S] = nullptr;
            tgraph_[S] = nullptr;
            targs_[S] = nullptr;
        }
    }
    void launch_step(cudaGraphExec_t* exec) {
        {
            for (size_t k = 0; k < m_.size(); k++)
                if (m_[k] && m_[k]->par_ != (par_ ^ d_[k]))
                    fail("batch: the cavities' states have diverged (a failed step); rebuild the batch");
            check(cudaGraphLaunch(exec[par_], stream_));
            for (S_* s : m_) {
                if (!s) continue;
                if (s->pending_.empty()) s->steps_before_ = s->hc_.steps;
                s->pending_.push_back(s->par_);
                s->par_ ^= 1;
                s->tail_queued_ = false;          // a batch step has no per-cavity tail: sync reads the control block
                s->probes_fresh_ = false;
            }
            par_ ^= 1;
            queued_ = true;
        }
    }

public:
    // waits for the queued steps; every occupied slot's report (its last good state if it failed; an empty
    // slot's report is zero with steps = -1), then the first failure as an error naming the slot
    void sync(CavityReport* reports) override {
        check(cudaStreamSynchronize(stream_));
        queued_ = false;
        std::string first;
        for (size_t i = 0; i < m_.size(); i++) {
            if (!m_[i]) {
                if (reports) {
                    std::memset(&reports[i], 0, sizeof(CavityReport));
                    reports[i].steps = -1;
                }
                continue;
            }
            try {
                m_[i]->sync(reports ? &reports[i] : nullptr);
            } catch (const std::exception& e) {
                if (first.empty()) first = "cavity " + std::to_string(i) + ": " + e.what();
                if (reports) m_[i]->report(&reports[i]);
            }
        }
        if (!first.empty()) fail(first);
    }
    // Put cavity `s` into slot `slot` (nullptr: empty the slot) without rebuilding the step graphs: its
    // argument records for both graphs and the slot's live flag are written into the device buffers the graphs
    // read.  A newly placed cavity need not be at the batch's state parity (the slot keeps the offset).
    void set_member(int slot, SolverBase* base) override {
        if (slot < 0 || slot >= (int)m_.size()) fail("batch: slot out of range");
        if (queued_) fail("batch: steps are queued; sync first");
        S_* s = nullptr;
        if (base) {
            s = dynamic_cast<S_*>(base);
            if (!s) fail("batch: the cavity's precision form differs from the batch's");
            for (size_t k = 0; k < m_.size(); k++)
                if (m_[k] == s && (int)k != slot) fail("batch: the cavity is already in another slot");
            check_member(s, *s);
            if (s->nx_ != nx_ || s->ny_ != ny_ || s->nz_ != nz_) fail("batch: the cavity's grid size differs from the batch's");
            if (s->tc_fdm_ != tc_fdm_ || s->sweep_kind_ != sweep_kind_) fail("batch: the cavity's kernels differ from the batch's");
            d_[slot] = s->par_ ^ par_;
            for (int S = 0; S < 2; S++) {
                std::vector<LaunchRecord> rec;
                {
                    RecordGuard guard(&rec, (int)m_.size(), dgemm_tile_, pairs_);
                    record_member(*s, S ^ d_[slot], S);
                }
                const Layout& L = layout_[S];
                if (rec.size() != L.launches.size()) fail("batch: the cavity's launch sequence differs from the batch's");
                for (size_t j = 0; j < rec.size(); j++) {
                    const LaunchSlot& ls = L.launches[j];
                    if (rec[j].kind != ls.kind || rec[j].variant != ls.variant || rec[j].smem != ls.smem ||
                        rec[j].args.size() != ls.size || rec[j].grid.x != ls.grid.x || rec[j].grid.y != ls.grid.y ||
                        rec[j].grid.z != ls.grid.z)
                        fail("batch: the cavity's launch sequence differs from the batch's");
                    std::memcpy(host_[S].data() + ls.off + (size_t)slot * ls.size, rec[j].args.data(), ls.size);
                }
            }
        }
        m_[slot] = s;
        for (int S = 0; S < 2; S++) {
            reinterpret_cast<int*>(host_[S].data() + layout_[S].live)[slot] = s ? 1 : 0;
            check(cudaMemcpyAsync(dargs_[S], host_[S].data(), host_[S].size(), cudaMemcpyHostToDevice, stream_));
        }
        check(cudaStreamSynchronize(stream_));
    }

private:
    struct RecordGuard {
        RecordGuard(std::vector<LaunchRecord>* r, int batch, int dgemm_tile, int pairs) {
            g_launch_record = r;
            g_launch_batch = batch;
            g_dgemm_tile = dgemm_tile;
            g_batch_pairs = pairs;
        }
        ~RecordGuard() {
            g_launch_record = nullptr;
            g_launch_batch = 1;
            g_dgemm_tile = 0;
            g_batch_pairs = -1;
        }
    };
    static size_t align256(size_t n) { return (n + 255) / 256 * 256; }
    static void check_member(const S_* s, const S_& f) {
        if (s->tc_fdm_ != f.tc_fdm_ || s->sweep_kind_ != f.sweep_kind_ || s->sweep_kind_ == kSweepFace)
            fail("batch: every cavity needs the same kernels (march or tile sweep)");
        if (s->eager_) fail("batch: not available with CAVITY_GRAPHS=0");
        if (!s->pending_.empty()) fail("batch: a cavity has queued steps; sync it first");
    }

    // where one recorded launch's argument records sit in the argument buffer of a graph
    struct LaunchSlot {
        int kind, variant;
        size_t smem, off, size;
        dim3 grid;
    };
    struct Layout {
        std::vector<LaunchSlot> launches;
        size_t live = 0;                       // the slots' live flags (int each)
    };

    // The launches of one cavity's step, for the cavity's state parity Sm inside the graph of batch parity S
    // (whose while-node handles the loop kernels set), in the order the graph runs them.  `part` selects one
    // piece of the sequence (see sequence); -1 all of them.
    void member_part(S_& s, int Sm, int S, int stage, int part) {
        const int Xs = Sm ^ 1, Ys = 2;
        const int in = stage == 0 ? Sm : stage == 1 ? Xs : Ys;
        const int out = stage == 1 ? Ys : Xs;
        const int cur = stage == 1 ? Xs : Ys;
        const cudaGraphConditionalHandle h = handles_[S][stage];
        cudaStream_t st = part == 3 ? body_stream_ : stream_;
        switch (part) {
        case 0: s.launch_momentum(st, stage, Sm, in, out); break;
        case 1: s.launch_start(st, s.M_[out], true, stage, Sm, cur, h, 2); break;
        case 2:
        case 3: s.launch_pass(st, s.praw_, h, 2); break;
        case 4: s.launch_finish(st, s.M_[out], s.U_[out], s.PHI_[out], true, stage, stage == 2); break;
        }
    }
    void record_member(S_& s, int Sm, int S) {
        s.launch_step_begin(stream_);
        for (int stage = 0; stage < 3; stage++)
            for (int part = 0; part < 5; part++) member_part(s, Sm, S, stage, part);
    }

    // run `fn(member, slot)` on every slot (an empty slot records the first member: its records are never read,
    // the slot being dead) with a recorder installed, append the argument records of each recorded launch to
    // `host` (one contiguous array per launch, slot after slot) and, when `launch`, issue the batched launches
    template <class F> void emit(cudaStream_t st, F fn, std::vector<unsigned char>& host, Layout& L, bool launch) {
        const size_t B = m_.size();
        std::vector<std::vector<LaunchRecord>> recs(B);
        for (size_t b = 0; b < B; b++) {
            RecordGuard guard(&recs[b], (int)B, dgemm_tile_, pairs_);
            if (m_[b]) fn(*m_[b], (int)b);
            else fn(*proto_, 0);
        }
        for (size_t b = 1; b < B; b++) {
            bool same = recs[b].size() == recs[0].size();
            for (size_t j = 0; same && j < recs[0].size(); j++) {
                const LaunchRecord &x = recs[0][j], &y = recs[b][j];
                same = x.kind == y.kind && x.variant == y.variant && x.smem == y.smem && x.args.size() == y.args.size();
            }
            if (!same) fail("batch: the cavities' launch sequences differ");
        }
        const unsigned char* dbase = static_cast<const unsigned char*>(dargs_cur_);
        for (size_t j = 0; j < recs[0].size(); j++) {
            const size_t sz = recs[0][j].args.size();
            const size_t off = align256(host.size());
            host.resize(off + sz * B);
            for (size_t b = 0; b < B; b++) std::memcpy(host.data() + off + b * sz, recs[b][j].args.data(), sz);
            L.launches.push_back({recs[0][j].kind, recs[0][j].variant, recs[0][j].smem, off, sz, recs[0][j].grid});
            // the work list: every slot's blocks of its cavity's own launch grid, slot after slot (identical
            // lists are stored once)
            size_t items_off = 0, n_items = 0;
            if (recs[0][j].kind != kLkStepBegin) {
                std::vector<BatchItem> items;
                for (size_t b = 0; b < B; b++) {
                    const dim3 g = recs[b][j].grid;
                    for (unsigned int z = 0; z < g.z; z++)
                        for (unsigned int y = 0; y < g.y; y++)
                            for (unsigned int x = 0; x < g.x; x++) items.push_back({(unsigned int)b, x, y, z, g.x, g.y, g.z, 0u});
                }
                std::string key(reinterpret_cast<const char*>(items.data()), items.size() * sizeof(BatchItem));
                auto it = item_lists_.find(key);
                if (it == item_lists_.end()) {
                    items_off = align256(host.size());
                    host.resize(items_off + key.size());
                    std::memcpy(host.data() + items_off, key.data(), key.size());
                    item_lists_.emplace(std::move(key), items_off);
                } else {
                    items_off = it->second;
                }
                n_items = items.size();
            }
            if (launch)
                launch_batched(recs[0][j], dbase + off, reinterpret_cast<const BatchItem*>(dbase + items_off),
                               (unsigned int)n_items, reinterpret_cast<const int*>(dbase + L.live), (int)B, st);
        }
    }
    void launch_batched(const LaunchRecord& r, const void* d, const BatchItem* items, unsigned int n_items,
                        const int* live, int B, cudaStream_t st) {
        const dim3 g(n_items);
        switch (r.kind) {
        case kLkStepBegin:
            check(launch_pdl(step_begin_batched, dim3(1, 1, B), dim3(32), 0, st, (const StepBeginArgs*)d, live));
            break;
        case kLkSweep:
            if (r.variant == kSweepMarch)
                check(launch_pdl(sweep_march_batched<T, S_::kMarchTX, S_::kMarchTY>, g, dim3(S_::MarchG::NT), r.smem, st,
                                 (const MomentumArgs<T>*)d, items, live));
            else if (r.variant == kSweepPair) {
                if constexpr (sizeof(T) == 4)
                    check(launch_pdl(sweep_pair_batched<kTY, kTZ, S_::kPairNT>, g, dim3(S_::kPairNT), r.smem, st,
                                     (const MomentumArgs<T>*)d, items, live));
                else
                    fail("the packed sweep is FP32 only");
            } else
                check(launch_pdl(sweep_tile_batched<T, kTY, kTZ, kNT>, g, dim3(kNT), r.smem, st,
                                 (const MomentumArgs<T>*)d, items, live));
            break;
        case kLkStart:
            check(launch_pdl(projection_start_batched<T>, g, dim3(kThreads), 0, st, (const StartArgs<T>*)d, items, live));
            break;
        case kLkResidual:
            check(launch_pdl(residual_batched, g, dim3(kThreads), 0, st, (const ResidualArgs*)d, items, live));
            break;
        case kLkFinish:
            check(launch_pdl(finish_batched<T>, g, dim3(kThreads), 0, st, (const FinishArgs<T>*)d, items, live));
            break;
        case kLkDgemm64:
            check(launch_pdl(dgemm_mma_batched<64, 64, 2, 2, 32>, g, dim3(128), 0, st, (const GemmArgs<double>*)d, items,
                             live));
            break;
        case kLkDgemm32:
            check(launch_pdl(dgemm_mma_batched<32, 32, 2, 4, 64>, g, dim3(256), 0, st, (const GemmArgs<double>*)d, items,
                             live));
            break;
        case kLkTc: launch_tc_batched(r.variant, g, items, live, (const TcTransformArgs*)d, st); break;
        case kLkPair: launch_pair_batched(r.variant, g, items, live, (const FdmPairArgs*)d, st); break;
        default: fail("batch: unknown launch");
        }
    }
    // the step of batch parity S (as Solver::enqueue_step, each slot at its own state parity S ^ d); `launch` =
    // false only records (sizes the argument buffer), true captures the batched launches into the graph being
    // built on stream_
    void sequence(int S, std::vector<unsigned char>& host, Layout& L, bool launch, bool timing = false) {
        // timing: events before and after the parts of each stage outside the refinement loop (part_times)
        auto mark = [&](int stage, int part, int end) {
            if (timing && launch)
                check(cudaEventRecordWithFlags(tev_[(stage * kParts + part) * 2 + end], stream_, cudaEventRecordExternal));
        };
        L.live = 0;
        host.resize(align256(sizeof(int) * m_.size()));
        for (size_t i = 0; i < m_.size(); i++) reinterpret_cast<int*>(host.data())[i] = m_[i] ? 1 : 0;
        auto par = [&](int b) { return S ^ d_[b]; };
        emit(stream_, [&](S_& s, int) { s.launch_step_begin(stream_); }, host, L, launch);
        for (int stage = 0; stage < 3; stage++) {
            mark(stage, 0, 0);
            emit(stream_, [&](S_& s, int b) { member_part(s, par(b), S, stage, 0); }, host, L, launch);
            mark(stage, 0, 1);
            cudaGraph_t g = nullptr;
            const cudaGraphNode_t* deps = nullptr;
            size_t ndeps = 0;
            cudaStreamCaptureStatus status;
            if (launch) {
                check(cudaStreamGetCaptureInfo(stream_, &status, nullptr, &g, &deps, &ndeps));
                check(cudaGraphConditionalHandleCreate(&handles_[S][stage], g, 0, cudaGraphCondAssignDefault));
            }
            mark(stage, 1, 0);
            emit(stream_, [&](S_& s, int b) { member_part(s, par(b), S, stage, 1); }, host, L, launch);
            mark(stage, 1, 1);
            // the first pass outside the loop (see Solver::captured_loop), then the loop
            mark(stage, 2, 0);
            emit(stream_, [&](S_& s, int b) { member_part(s, par(b), S, stage, 2); }, host, L, launch);
            mark(stage, 2, 1);
            if (launch) {
                check(cudaStreamGetCaptureInfo(stream_, &status, nullptr, &g, &deps, &ndeps));
                cudaGraphNodeParams cp = {cudaGraphNodeTypeConditional};
                cp.type = cudaGraphNodeTypeConditional;
                cp.conditional.handle = handles_[S][stage];
                cp.conditional.type = cudaGraphCondTypeWhile;
                cp.conditional.size = 1;
                cudaGraphNode_t node;
                check(cudaGraphAddNode(&node, g, deps, ndeps, &cp));
                cudaGraph_t body = cp.conditional.phGraph_out[0];
                check(cudaStreamBeginCaptureToGraph(body_stream_, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed));
                emit(body_stream_, [&](S_& s, int b) { member_part(s, par(b), S, stage, 3); }, host, L, launch);
                check(cudaStreamEndCapture(body_stream_, &body));
                check(cudaStreamUpdateCaptureDependencies(stream_, &node, 1, cudaStreamSetCaptureDependencies));
            } else {
                emit(stream_, [&](S_& s, int b) { member_part(s, par(b), S, stage, 3); }, host, L, launch);
            }
            mark(stage, 3, 0);
            emit(stream_, [&](S_& s, int b) { member_part(s, par(b), S, stage, 4); }, host, L, launch);
            mark(stage, 3, 1);
        }
    }
    // the step graph of batch parity S; with `timing` the instrumented twin (part_times), built from the current
    // members with its own argument buffer and refinement-loop handles (the plain graph's are kept)
    void build(int S, bool timing = false) {
        if (timing) {
            cudaGraphConditionalHandle saved[3] = {handles_[S][0], handles_[S][1], handles_[S][2]};
            std::vector<unsigned char> host;
            Layout L;
            item_lists_.clear();
            sequence(S, host, L, false);
            check(cudaMalloc(&targs_[S], std::max<size_t>(host.size(), 256)));
            dargs_cur_ = targs_[S];
            host.clear();
            item_lists_.clear();
            L = Layout();
            check(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal));
            sequence(S, host, L, true, true);
            check(cudaStreamEndCapture(stream_, &tgraph_[S]));
            check(cudaGraphInstantiate(&texec_[S], tgraph_[S], 0));
            check(cudaMemcpy(targs_[S], host.data(), host.size(), cudaMemcpyHostToDevice));
            for (int k = 0; k < 3; k++) handles_[S][k] = saved[k];
            dargs_cur_ = dargs_[S];
            return;
        }
        std::vector<unsigned char> host;
        Layout L;
        item_lists_.clear();
        sequence(S, host, L, false);
        check(cudaMalloc(&dargs_[S], std::max<size_t>(host.size(), 256)));
        dargs_cur_ = dargs_[S];
        host.clear();
        item_lists_.clear();
        layout_[S] = Layout();
        check(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal));
        sequence(S, host, layout_[S], true);
        check(cudaStreamEndCapture(stream_, &graph_[S]));
        check(cudaGraphInstantiate(&exec_[S], graph_[S], 0));
        check(cudaMemcpy(dargs_[S], host.data(), host.size(), cudaMemcpyHostToDevice));
        host_[S] = std::move(host);
    }

    std::vector<S_*> m_;                      // slot -> cavity (nullptr: empty)
    std::vector<int> d_;                      // slot -> its cavity's state parity relative to the batch's
    S_* proto_ = nullptr;                     // a member, while the graphs are built
    int par_ = 0;                             // the batch's state parity: the graph the next step launches
    bool queued_ = false;
    int nx_ = 0, ny_ = 0, nz_ = 0, sweep_kind_ = 0;
    bool tc_fdm_ = false;
    cudaStream_t stream_ = nullptr, body_stream_ = nullptr;
    cudaGraph_t graph_[2] = {nullptr, nullptr}, tgraph_[2] = {nullptr, nullptr};
    cudaGraphExec_t exec_[2] = {nullptr, nullptr}, texec_[2] = {nullptr, nullptr};
    cudaEvent_t tev_[3 * kParts * 2] = {};
    void* targs_[2] = {nullptr, nullptr};     // argument buffers of the timing graphs
    cudaGraphConditionalHandle handles_[2][3] = {};
    void* dargs_[2] = {nullptr, nullptr};
    void* dargs_cur_ = nullptr;
    std::vector<unsigned char> host_[2];      // host copies of the argument buffers
    Layout layout_[2];
    bool mixed_sizes_ = false;
    int pairs_ = 0;             // FP64 passes as paired launches (every member's axes at most 64 cells)
    int dgemm_tile_ = 0;
    std::map<std::string, size_t> item_lists_;      // work lists already in the argument buffer, by content
};

static SolverBase* make_solver(const CavityConfig& c, int precision) {
    if (precision == 0) return new Solver<double>(c);
    if (precision == 1) return new Solver<float>(c);
    fail("precision must be 0 (fp64) or 1 (mixed)");
}

// bytes a cavity would hold: 3 sets x (3 face arrays x 2) + m0 of T, 14 cell arrays of double, tables
static long long estimate_bytes(const CavityConfig& c, int precision) {
    const long long nx = c.nx, ny = c.ny, nz = c.nz, cells = nx * ny * nz;
    const long long faces = (nx + 1) * ny * nz + nx * (ny + 1) * nz + nx * ny * (nz + 1);
    const long long fb = precision == 0 ? 8 : 4;
    const long long maxface = std::max((nx + 1) * ny * nz, nx * ny * (nz + 1));
    const long long tc = precision == 1 && nx % 4 == 0
                             ? 4 * cells + 4 * 4 * (cavity::basis_image_floats((int)nx, (int)nx) +
                                                    cavity::basis_image_floats((int)ny, (int)ny) +
                                                    cavity::basis_image_floats((int)nz, (int)nz))
                             : 0;
    return 7 * faces * fb + 16 * cells * 8 + 2 * 8 * maxface + 4 * std::max(maxface, 2 * cells) +
           2 * 8 * (nx * nx + ny * ny + nz * nz) + 64 * (maxface / 256 + 8) + tc + (1 << 20);
}

// One FDM pass of the mixed form on the tensor cores on caller-provided device arrays, with the reference's
// scaling of r to rms 1 and float S and 1/lambda (backend.cu:766-814); every intermediate is allocated on the
// stream.
static void fdm_pass_tf32(int nx, int ny, int nz, const double* const s[3], const double* const st[3],
                          const double* inv_lambda, const double* r, double* phi, cudaStream_t stream) {
    if (nx < 1 || ny < 1 || nz < 1 || nx > 1024 || ny > 1024 || nz > 1024) fail("fdm pass: 1 <= nx, ny, nz <= 1024");
    if (nx % 4) fail("fdm pass (tensor cores): nx must be a multiple of 4");
    if (!inv_lambda || !r || !phi) fail("fdm pass: null pointer");
    for (int a = 0; a < 3; a++)
        if (!s[a] || !st[a]) fail("fdm pass: null eigenbasis");
    const long long n = (long long)nx * ny * nz;
    const int dims[3] = {nx, ny, nz};
    int dev = 0, sms = 148;
    check(cudaGetDevice(&dev));
    check(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    check(tc_transform_prepare());
    std::vector<void*> owned;
    auto alloc = [&](size_t bytes) {
        void* p = nullptr;
        check(cudaMallocAsync(&p, bytes, stream));
        owned.push_back(p);
        return p;
    };
    float* t1 = (float*)alloc(sizeof(float) * n);
    float* t2 = (float*)alloc(sizeof(float) * n);
    float* invf = (float*)alloc(sizeof(float) * n);
    Control* c = (Control*)alloc(sizeof(Control));
    TcFdmOperands op;
    op.nx = nx; op.ny = ny; op.nz = nz;
    op.inv_lambda = invf;
    for (int a = 0; a < 3; a++) {
        float* img[4];
        for (int i = 0; i < 4; i++) img[i] = (float*)alloc(sizeof(float) * basis_image_floats(dims[a], dims[a]));
        launch_basis_image(stream, s[a], dims[a], 0, img[0], img[1]);
        launch_basis_image(stream, s[a], dims[a], 1, img[2], img[3]);
        for (int i = 0; i < 4; i++) op.img[a][i] = img[i];
    }
    const Control hc = standalone_fdm_control();
    check(cudaMemcpyAsync(c, &hc, sizeof hc, cudaMemcpyHostToDevice, stream));
    control_norm_kernel<<<1, kThreads, 0, stream>>>(r, n, c);
    convert_kernel<double, float><<<blocks_for(n), kThreads, 0, stream>>>(inv_lambda, invf, n);
    launch_tc_fdm_pass(stream, op, r, nullptr, phi, t1, t2, c, 0, false, sms);
    const cudaError_t launched = cudaGetLastError();
    Control out;
    const cudaError_t copied = cudaMemcpyAsync(&out, c, sizeof out, cudaMemcpyDeviceToHost, stream);
    for (void* p : owned) check(cudaFreeAsync(p, stream));
    check(launched);
    check(copied);
    check(cudaStreamSynchronize(stream));
    if (out.error == kDeviceWait) fail("fdm pass (tensor cores): a transform timed out waiting for its MMAs");
}

// One FDM pass on caller-provided device arrays; the two intermediates are allocated on the stream.
static void fdm_pass(int nx, int ny, int nz, const double* const s[3], const double* const st[3],
                     const double* inv_lambda, const double* r, double* phi, cudaStream_t stream) {
    if (nx < 1 || ny < 1 || nz < 1 || nx > 1024 || ny > 1024 || nz > 1024) fail("fdm pass: 1 <= nx, ny, nz <= 1024");
    if (!inv_lambda || !r || !phi) fail("fdm pass: null pointer");
    FdmOperands op;
    op.nx = nx; op.ny = ny; op.nz = nz;
    for (int a = 0; a < 3; a++) {
        if (!s[a] || !st[a]) fail("fdm pass: null eigenbasis");
        op.s[a] = s[a];
        op.st[a] = st[a];
    }
    op.inv_lambda = inv_lambda;
    const size_t n = (size_t)nx * ny * nz;
    double *t1 = nullptr, *t2 = nullptr;
    Control* c = nullptr;
    check(cudaMallocAsync((void**)&t1, sizeof(double) * n, stream));
    check(cudaMallocAsync((void**)&t2, sizeof(double) * n, stream));
    check(cudaMallocAsync((void**)&c, sizeof(Control), stream));
    const Control hc = standalone_fdm_control();
    check(cudaMemcpyAsync(c, &hc, sizeof hc, cudaMemcpyHostToDevice, stream));
    check(pair_prepare());
    launch_fdm_pass(stream, op, r, nullptr, phi, t1, t2, c, 0, false, pass_form_from_env());
    const cudaError_t launched = cudaGetLastError();
    check(cudaFreeAsync(t1, stream));
    check(cudaFreeAsync(t2, stream));
    check(cudaFreeAsync(c, stream));
    check(launched);
    check(cudaStreamSynchronize(stream));
}

// ------------------------------------------------------------------------------------------ no-allocation pass
// The FDM pass for callers that cannot allocate device memory: its two intermediates and its control block
// live in file-scope device arrays instead of cudaMallocAsync'd buffers.  Every GPU that loads the library
// holds these 4 MiB until the process exits; all calls on a device share them.
constexpr long long kNoAllocMaxCells = 262144;                      // 64^3
static __device__ __align__(256) double g_noalloc_transforms[2 * kNoAllocMaxCells];
static __device__ __align__(256) Control g_noalloc_control;

struct NoAllocScratch {
    double* transforms = nullptr;
    Control* control = nullptr;
};
static std::mutex g_noalloc_mutex;
static NoAllocScratch g_noalloc_scratch[64];                        // per device, filled on first use

// Device addresses of the arrays on the current device (host code cannot use their names as addresses).
static NoAllocScratch noalloc_scratch() {
    int dev = 0;
    check(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) fail("fdm pass (no allocation): device ordinal out of range");
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    NoAllocScratch& s = g_noalloc_scratch[dev];
    if (!s.transforms) {
        void* t = nullptr;
        void* c = nullptr;
        check(cudaGetSymbolAddress(&t, g_noalloc_transforms));
        check(cudaGetSymbolAddress(&c, g_noalloc_control));
        s.transforms = (double*)t;
        s.control = (Control*)c;
    }
    return s;
}

static void fdm_pass_noalloc(int nx, int ny, int nz, const double* const s[3], const double* const st[3],
                             const double* inv_lambda, const double* r, double* phi, cudaStream_t stream) {
    if (nx < 1 || ny < 1 || nz < 1 || nx > 1024 || ny > 1024 || nz > 1024)
        fail("fdm pass (no allocation): 1 <= nx, ny, nz <= 1024");
    const long long n = (long long)nx * ny * nz;
    if (n > kNoAllocMaxCells) {
        char msg[200];
        std::snprintf(msg, sizeof msg, "fdm pass (no allocation): %d x %d x %d = %lld cells exceeds the maximum of %lld",
                      nx, ny, nz, n, kNoAllocMaxCells);
        fail(msg);
    }
    if (!inv_lambda || !r || !phi) fail("fdm pass (no allocation): null pointer");
    FdmOperands op;
    op.nx = nx; op.ny = ny; op.nz = nz;
    for (int a = 0; a < 3; a++) {
        if (!s[a] || !st[a]) fail("fdm pass (no allocation): null eigenbasis");
        op.s[a] = s[a];
        op.st[a] = st[a];
    }
    op.inv_lambda = inv_lambda;
    const NoAllocScratch scratch = noalloc_scratch();
    // the control block keeps the previous call's contents: reset its flags (error, reset) to zero
    const Control hc = standalone_fdm_control();
    check(cudaMemcpyAsync(scratch.control, &hc, sizeof hc, cudaMemcpyHostToDevice, stream));
    check(pair_prepare());
    launch_fdm_pass(stream, op, r, nullptr, phi, scratch.transforms, scratch.transforms + n, scratch.control, 0, false,
                    pass_form_from_env());
    check(cudaGetLastError());
    check(cudaStreamSynchronize(stream));
}

}  // namespace cavity

// ================================================================================================ C ABI
using cavity::SolverBase;
struct CavitySolver { std::unique_ptr<SolverBase> s; };
struct CavityBatch { std::unique_ptr<cavity::BatchBase> b; };

static thread_local std::string g_last_error;     // per calling thread (cavities set up on a worker thread)
static CavitySolver* g_default = nullptr;
static int g_precision = 0;

template <class F> static int safely(F f) {
    try {
        f();
        return 0;
    } catch (const std::exception& e) {
        g_last_error = e.what();
        return 1;
    }
}
static SolverBase& S() {
    if (!g_default) cavity::fail("no solver: call solver_create first");
    return *g_default->s;
}
static SolverBase& H(CavitySolver* h) {
    if (!h || !h->s) cavity::fail("invalid solver handle");
    return *h->s;
}

extern "C" {
int solver_destroy(void) {
    return safely([&] {
        delete g_default;
        g_default = nullptr;
    });
}
int solver_create(const CavityConfig* config) {
    return safely([&] {
        delete g_default;
        g_default = nullptr;
        std::unique_ptr<CavitySolver> h(new CavitySolver);
        h->s.reset(cavity::make_solver(*config, g_precision));
        g_default = h.release();
    });
}
int solver_initialize(const double* v, const double* w) { return safely([&] { S().initialize(v, w); }); }
int solver_step(CavityReport* r) { return safely([&] { S().step(r); }); }
int solver_kick(const double* nu, const double* nv, const double* nw, double amp, int passes) {
    return safely([&] { const double* n[3] = {nu, nv, nw}; S().kick(n, amp, passes); });
}
int solver_report(CavityReport* r) { return safely([&] { S().report(r); }); }
int solver_diagnostics(CavityDiagnostics* d) { return safely([&] { S().diagnostics(d); }); }
int solver_grid(int axis, double* faces, double* centres) { return safely([&] { S().grid(axis, faces, centres); }); }
int solver_get_field(int field, void* out) { return safely([&] { S().get_field(field, out); }); }
int solver_set_field(int field, const void* in) { return safely([&] { S().set_field(field, in); }); }
int solver_set_clock(double t, long long steps, double last_dt) { return safely([&] { S().set_clock(t, steps, last_dt); }); }
int solver_probes(float* out) { return safely([&] { S().probes(out); }); }
int solver_add_statistics(double weight, double* centreline) { return safely([&] { S().add_statistics(weight, centreline); }); }
int solver_get_statistics(double* sums) { return safely([&] { S().get_statistics(sums); }); }
int solver_set_statistics(const double* sums) { return safely([&] { S().set_statistics(sums); }); }
int solver_midplane(float* out) { return safely([&] { S().midplane(out); }); }
int solver_q_volume(int colour_w, float* q, float* colour) { return safely([&] { S().q_volume(colour_w, q, colour); }); }
const char* solver_last_error(void) { return g_last_error.c_str(); }

int cavity_get_field_f64(int field, double* out) { return safely([&] { S().get_field_f64(field, out); }); }
int cavity_set_precision(int precision) {
    return safely([&] {
        if (precision != 0 && precision != 1) cavity::fail("precision must be 0 (fp64) or 1 (mixed)");
        g_precision = precision;
    });
}
int cavity_create(const CavityConfig* config, int precision, CavitySolver** out) {
    return safely([&] {
        std::unique_ptr<CavitySolver> h(new CavitySolver);
        h->s.reset(cavity::make_solver(*config, precision));
        *out = h.release();
    });
}
int cavity_destroy(CavitySolver* s) {
    return safely([&] {
        if (s == g_default) g_default = nullptr;
        delete s;
    });
}
int cavity_initialize(CavitySolver* s, const double* v, const double* w) { return safely([&] { H(s).initialize(v, w); }); }
int cavity_step(CavitySolver* s, CavityReport* r) { return safely([&] { H(s).step(r); }); }
int cavity_step_async(CavitySolver* s, int count) { return safely([&] { H(s).step_async(count); }); }
int cavity_sync(CavitySolver* s, CavityReport* r) { return safely([&] { H(s).sync(r); }); }
int cavity_get_field(CavitySolver* s, int field, void* out) { return safely([&] { H(s).get_field(field, out); }); }
int cavity_report(CavitySolver* s, CavityReport* r) { return safely([&] { H(s).report(r); }); }
int cavity_set_clock(CavitySolver* s, double t, long long steps, double last_dt) {
    return safely([&] { H(s).set_clock(t, steps, last_dt); });
}
int cavity_set_field(CavitySolver* s, int field, const void* in) { return safely([&] { H(s).set_field(field, in); }); }
int cavity_probes(CavitySolver* s, float* out) { return safely([&] { H(s).probes(out); }); }
int cavity_add_statistics(CavitySolver* s, double weight, double* centreline) {
    return safely([&] { H(s).add_statistics(weight, centreline); });
}
int cavity_get_statistics(CavitySolver* s, double* sums) { return safely([&] { H(s).get_statistics(sums); }); }
int cavity_diagnostics(CavitySolver* s, CavityDiagnostics* d) { return safely([&] { H(s).diagnostics(d); }); }
long long cavity_device_bytes(const CavitySolver* s) { return s && s->s ? s->s->device_bytes() : -1; }
long long cavity_estimate_bytes(const CavityConfig* config, int precision) {
    return cavity::estimate_bytes(*config, precision);
}
int cavity_time_steps(CavitySolver* s, int warmup, int steps, int flush_l2, float* ms, float* kms) {
    return safely([&] { H(s).time_steps(warmup, steps, flush_l2, ms, kms); });
}
int cavity_autotune(CavitySolver* s, int steps, int* march_chunks, int* dgemm_tile, int* fused_pass, float* ms_per_step) {
    return safely([&] { H(s).autotune(steps, march_chunks, dgemm_tile, fused_pass, ms_per_step); });
}
int cavity_kernel_times(CavitySolver* s, double* ms) {
    return safely([&] { H(s).kernel_times(ms); });
}
CavitySolver* cavity_default(void) { return g_default; }
int cavity_step_outputs_async(CavitySolver* s, int count, int statistics) {
    return safely([&] { H(s).step_outputs_async(count, statistics); });
}
int cavity_sync_outputs(CavitySolver* s, CavityReport* r, float* probes, int max_steps, int* steps_out) {
    return safely([&] {
        const int n = H(s).sync_outputs(r, probes, max_steps);
        if (steps_out) *steps_out = n;
    });
}
long long cavity_checkpoint_bytes(const CavitySolver* s) { return s && s->s ? s->s->checkpoint_bytes() : -1; }
int cavity_checkpoint_save(CavitySolver* s, void* dst, int dst_is_device) {
    return safely([&] {
        if (!dst) cavity::fail("checkpoint: null buffer");
        H(s).checkpoint_save(dst, dst_is_device);
    });
}
int cavity_checkpoint_load(CavitySolver* s, const void* src, int src_is_device) {
    return safely([&] {
        if (!src) cavity::fail("checkpoint: null buffer");
        H(s).checkpoint_load(src, src_is_device);
    });
}
int cavity_kernels_per_step(const CavitySolver* s, int passes) { return s && s->s ? s->s->kernels_per_step(passes) : -1; }
int cavity_fdm_pass(int nx, int ny, int nz, const double* const s[3], const double* const st[3],
                    const double* inv_lambda, const double* r, double* phi, void* stream) {
    return safely([&] { cavity::fdm_pass(nx, ny, nz, s, st, inv_lambda, r, phi, (cudaStream_t)stream); });
}
int cavity_fdm_pass_tf32(int nx, int ny, int nz, const double* const s[3], const double* const st[3],
                         const double* inv_lambda, const double* r, double* phi, void* stream) {
    return safely([&] { cavity::fdm_pass_tf32(nx, ny, nz, s, st, inv_lambda, r, phi, (cudaStream_t)stream); });
}
int cavity_fdm_pass_noalloc(int nx, int ny, int nz, const double* const s[3], const double* const st[3],
                            const double* inv_lambda, const double* r, double* phi, void* stream) {
    return safely([&] { cavity::fdm_pass_noalloc(nx, ny, nz, s, st, inv_lambda, r, phi, (cudaStream_t)stream); });
}
int cavity_eigenbasis(const CavityConfig* config, int axis, int on_gpu, double* lambda, double* S) {
    return safely([&] {
        if (!config || axis < 0 || axis > 2 || !lambda || !S) throw std::runtime_error("cavity_eigenbasis: bad arguments");
        const CavityConfig& c = *config;
        const int n = axis == 0 ? c.nx : axis == 1 ? c.ny : c.nz;
        if (n < 2) throw std::runtime_error("cavity_eigenbasis: an axis needs at least 2 cells");
        const cavity::AxisGrid g = cavity::make_axis_grid(c, n, axis == 2 ? n * (c.lz / n) : c.length);
        const cavity::AxisEigen e = on_gpu ? cavity::axis_eigen_gpu(g) : cavity::axis_eigen(g);
        std::memcpy(lambda, e.lambda.data(), sizeof(double) * n);
        std::memcpy(S, e.S.data(), sizeof(double) * n * n);
    });
}
long long cavity_pressure_passes(const CavitySolver* s) { return s && s->s ? s->s->pressure_passes() : -1; }
int cavity_batch_create(CavitySolver* const* members, int count, CavityBatch** out) {
    return cavity_batch_create_slots(members, count, count, out);
}
int cavity_batch_create_slots(CavitySolver* const* members, int count, int capacity, CavityBatch** out) {
    return safely([&] {
        if (!members || count < 1 || !out) cavity::fail("batch: need at least one cavity");
        std::vector<cavity::Solver<double>*> d;
        std::vector<cavity::Solver<float>*> f;
        for (int i = 0; i < count; i++) {
            SolverBase* s = &H(members[i]);
            if (auto* p = dynamic_cast<cavity::Solver<double>*>(s)) d.push_back(p);
            else if (auto* q = dynamic_cast<cavity::Solver<float>*>(s)) f.push_back(q);
        }
        if (!d.empty() && !f.empty()) cavity::fail("batch: every cavity needs the same precision form");
        std::unique_ptr<CavityBatch> b(new CavityBatch);
        if (!d.empty()) b->b.reset(new cavity::Batch<double>(d, capacity));
        else b->b.reset(new cavity::Batch<float>(f, capacity));
        *out = b.release();
    });
}
int cavity_batch_step_async(CavityBatch* b, int count) {
    return safely([&] {
        if (!b || !b->b) cavity::fail("invalid batch handle");
        b->b->step_async(count);
    });
}
int cavity_batch_sync(CavityBatch* b, CavityReport* reports) {
    return safely([&] {
        if (!b || !b->b) cavity::fail("invalid batch handle");
        b->b->sync(reports);
    });
}
int cavity_batch_set_member(CavityBatch* b, int slot, CavitySolver* s) {
    return safely([&] {
        if (!b || !b->b) cavity::fail("invalid batch handle");
        b->b->set_member(slot, s ? &H(s) : nullptr);
    });
}
int cavity_batch_size(const CavityBatch* b) { return b && b->b ? b->b->size() : -1; }
int cavity_batch_part_times(CavityBatch* b, int steps, double* ms) {
    return safely([&] {
        if (!b || !b->b || !ms || steps < 1) cavity::fail("batch part times: null batch or output, or steps < 1");
        b->b->part_times(steps, ms);
    });
}
int cavity_batch_destroy(CavityBatch* b) { return safely([&] { delete b; }); }
const char* cavity_last_error(void) { return g_last_error.c_str(); }
}
