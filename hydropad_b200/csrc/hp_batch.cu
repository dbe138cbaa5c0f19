// hp_batch.cu -- batches of boxes: the ensemble and the serving engine.
//
// Every member is an ordinary context (hp_ctx) whose state stays where
// hp_init put it.  A step of the batch runs, for each of the three sweep
// slots of evolve_sys, one persistent sweep launch per axis that some
// member sweeps in that slot (members at different nrot sweep different
// axes), then one timedet thread per member.  The launches read a table of
// per-(member, slot, axis) sweep arguments and a per-step plan listing, per
// launch, the members and the first work item of each; both live in device
// memory.  Plans of steps where every member is at the same nrot are
// static (one per nrot) and those steps may be replayed from CUDA graphs;
// other plans are staged through a small ring of pinned buffers.
#include <cuda_runtime.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "../../include/hydropad_b200.h"
#include "hp_ctx.h"
#include "hp_device.cuh"
#include "hp_launch.h"
#include "hp_sweep.cuh"
#include "hp_sweep_launch.cuh"

namespace hp {
int launch_sweep_batch_fp64(const BatchLaunch& bl, int axis, int tile, cudaStream_t st);
int launch_sweep_batch_mixed(const BatchLaunch& bl, int axis, int tile, cudaStream_t st);

int launch_sweep_batch(const BatchLaunch& bl, int axis, int tile, int precision, cudaStream_t st) {
    return precision == HP_PREC_MIXED ? launch_sweep_batch_mixed(bl, axis, tile, st)
                                      : launch_sweep_batch_fp64(bl, axis, tile, st);
}
}  // namespace hp

namespace {

constexpr int kRing = 4;          // dynamic plans in flight
constexpr int kLaunches = 9;      // (slot, axis) launches of one step at most
constexpr int kMaxCapacity = 4096;

int cuda_fail(cudaError_t e) {
    if (e == cudaSuccess) return HP_OK;
    if (e == cudaErrorMemoryAllocation) return HP_ERR_OOM;
    return HP_ERR_CUDA;
}
#define HP_CUDA(x)                                   \
    do {                                             \
        cudaError_t e_ = (x);                        \
        if (e_ != cudaSuccess) return cuda_fail(e_); \
    } while (0)

// One launch of a step: sweep slot s along `axis` over plan entries
// [off, off + nent) (argument indices), followed by nent + 1 item offsets.
struct PlanLaunch {
    int s, axis, off, nent, nitems;
};
struct Plan {
    std::vector<int> ints;
    PlanLaunch L[kLaunches];
    int nl = 0;
};

inline int arg_index(int member, int s, int axis) { return member * 9 + s * 3 + axis; }

}  // namespace

struct hp_batch {
    int dev, precision, cap;
    cudaStream_t stream;
    std::vector<hp_ctx*> members;
    std::vector<int> base;         // sweep_count % 3 of each member when the tables were built
    int tile[3];
    bool tables_valid;
    hp::SweepArgs* d_args;         // [cap * 9]
    hp::SweepArgs* h_args;         // pinned staging
    hp::DevCtl** d_ctls;           // [cap]
    hp::DevCtl** h_ctls;
    int* d_counters;               // [kLaunches] work-queue heads
    int plan_ints;                 // ints per plan slot
    int* d_plans;                  // [(kRing + 6) * plan_ints]: dynamic ring, then one static plan per nrot
    int* h_plans;                  // pinned, same layout
    cudaEvent_t ring_ev[kRing];
    int ring_next;
    unsigned* d_status;            // [cap]
    unsigned* h_status;            // pinned [cap]
    Plan static_plan[6];
    cudaGraphExec_t graph[6];
    int graph_kernels[6];
    long long launches;
};

namespace {

void drop_graphs(hp_batch* b) {
    for (int r = 0; r < 6; ++r)
        if (b->graph[r]) {
            cudaGraphExecDestroy(b->graph[r]);
            b->graph[r] = nullptr;
        }
}

// Plan of one step, given each member's nrot.  Within a launch the members
// are ordered by decreasing pencil length, so the longest work items leave
// the queue first.
void build_plan(const hp_batch* b, const std::vector<int>& nrot, Plan& P) {
    P.ints.clear();
    P.nl = 0;
    const int n = (int)b->members.size();
    std::vector<int> sel;
    for (int s = 0; s < 3; ++s)
        for (int axis = 0; axis < 3; ++axis) {
            sel.clear();
            for (int m = 0; m < n; ++m)
                if (hp::kSweepOrder[nrot[m] - 1][s] == axis) sel.push_back(m);
            if (sel.empty()) continue;
            auto len = [&](int m) {
                const hp::Box& x = b->members[m]->box;
                return axis == 0 ? x.nx : (axis == 1 ? x.ny : x.nz);
            };
            std::stable_sort(sel.begin(), sel.end(), [&](int u, int v) { return len(u) > len(v); });
            const int P_ = hp::kTilePencils[axis][b->tile[axis]];
            PlanLaunch& L = P.L[P.nl++];
            L.s = s;
            L.axis = axis;
            L.off = (int)P.ints.size();
            L.nent = (int)sel.size();
            for (int m : sel) P.ints.push_back(arg_index(m, s, axis));
            int first = 0;
            for (int m : sel) {
                P.ints.push_back(first);
                const hp::Box& x = b->members[m]->box;
                const long long np = axis == 0 ? (long long)x.ny * x.nz
                                               : (axis == 1 ? (long long)x.nx * x.nz : (long long)x.nx * x.ny);
                first += (int)((np + P_ - 1) / P_);
            }
            P.ints.push_back(first);
            L.nitems = first;
        }
}

// Argument table, control-block list and static plans of the current
// members and tiles.  Runs between steps with the batch's stream idle.
int ensure_tables(hp_batch* b) {
    const int n = (int)b->members.size();
    bool stale = !b->tables_valid;
    for (int m = 0; m < n && !stale; ++m)
        if ((int)(b->members[m]->sweep_count % 3) != b->base[m]) stale = true;
    if (!stale) return HP_OK;
    HP_CUDA(cudaStreamSynchronize(b->stream));
    drop_graphs(b);
    b->base.assign(n, 0);
    for (int m = 0; m < n; ++m) {
        const hp_ctx* x = b->members[m];
        b->base[m] = (int)(x->sweep_count % 3);
        for (int s = 0; s < 3; ++s)
            for (int axis = 0; axis < 3; ++axis)
                b->h_args[arg_index(m, s, axis)] =
                    hp::make_sweep_args(x->box, axis, (b->base[m] + s) % 3, hp::step_flags(x->prm, s));
        b->h_ctls[m] = x->box.ctl;
    }
    if (n > 0) {
        HP_CUDA(cudaMemcpyAsync(b->d_args, b->h_args, sizeof(hp::SweepArgs) * 9 * n, cudaMemcpyHostToDevice,
                                b->stream));
        HP_CUDA(cudaMemcpyAsync(b->d_ctls, b->h_ctls, sizeof(hp::DevCtl*) * n, cudaMemcpyHostToDevice, b->stream));
    }
    std::vector<int> nrot(n);
    for (int r = 1; r <= 6; ++r) {
        std::fill(nrot.begin(), nrot.end(), r);
        build_plan(b, nrot, b->static_plan[r - 1]);
        const std::vector<int>& v = b->static_plan[r - 1].ints;
        int* h = b->h_plans + (size_t)(kRing + r - 1) * b->plan_ints;
        if (!v.empty()) {
            memcpy(h, v.data(), v.size() * sizeof(int));
            HP_CUDA(cudaMemcpyAsync(b->d_plans + (size_t)(kRing + r - 1) * b->plan_ints, h, v.size() * sizeof(int),
                                    cudaMemcpyHostToDevice, b->stream));
        }
    }
    HP_CUDA(cudaStreamSynchronize(b->stream));
    b->tables_valid = true;
    return HP_OK;
}

// Launches of one step from a plan whose ints are at dplan on the device.
// Returns the number of kernels or a negative error.
int enqueue_plan(hp_batch* b, const Plan& P, const int* dplan) {
    int kern = 0;
    if (cudaMemsetAsync(b->d_counters, 0, sizeof(int) * kLaunches, b->stream) != cudaSuccess) return HP_ERR_CUDA;
    for (int l = 0; l < P.nl; ++l) {
        const PlanLaunch& L = P.L[l];
        hp::BatchLaunch bl;
        bl.args = b->d_args;
        bl.ent = dplan + L.off;
        bl.nent = L.nent;
        bl.nitems = L.nitems;
        bl.counter = b->d_counters + l;
        int k = hp::launch_peak_prepass_batch(bl, L.axis, b->stream);
        if (k < 0) return HP_ERR_CUDA;
        kern += k;
        k = hp::launch_sweep_batch(bl, L.axis, b->tile[L.axis], b->precision, b->stream);
        if (k < 0) return HP_ERR_CUDA;
        kern += k;
    }
    const int k = hp::launch_timedet_batch(b->d_ctls, (int)b->members.size(), b->stream);
    if (k < 0) return HP_ERR_CUDA;
    return kern + k;
}

}  // namespace

extern "C" {

int hp_batch_create(hp_batch** out, int device, int precision, int capacity) {
    if (!out) return HP_ERR_ARG;
    *out = nullptr;
    if (capacity < 1 || capacity > kMaxCapacity) return HP_ERR_ARG;
    if (precision != HP_PREC_FP64 && precision != HP_PREC_MIXED) return HP_ERR_ARG;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) return HP_ERR_NO_DEVICE;
    HP_CUDA(cudaSetDevice(device));
    hp_batch* b = new hp_batch();
    b->dev = device;
    b->precision = precision;
    b->cap = capacity;
    b->stream = nullptr;
    b->tile[0] = b->tile[1] = b->tile[2] = 0;
    b->tables_valid = false;
    b->d_args = nullptr; b->h_args = nullptr;
    b->d_ctls = nullptr; b->h_ctls = nullptr;
    b->d_counters = nullptr;
    b->plan_ints = 6 * capacity + 2 * kLaunches + 16;
    b->d_plans = nullptr; b->h_plans = nullptr;
    for (int r = 0; r < kRing; ++r) b->ring_ev[r] = nullptr;
    b->ring_next = 0;
    b->d_status = nullptr; b->h_status = nullptr;
    for (int r = 0; r < 6; ++r) {
        b->graph[r] = nullptr;
        b->graph_kernels[r] = 0;
    }
    b->launches = 0;
    int rc = HP_OK;
    auto fail = [&](int code) {
        hp_batch_destroy(b);
        return code;
    };
    const size_t plans = (size_t)(kRing + 6) * b->plan_ints * sizeof(int);
    if ((rc = cuda_fail(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking))) != HP_OK) return fail(rc);
    if ((rc = cuda_fail(cudaMalloc(&b->d_args, sizeof(hp::SweepArgs) * 9 * capacity))) != HP_OK) return fail(rc);
    if ((rc = cuda_fail(cudaMallocHost(&b->h_args, sizeof(hp::SweepArgs) * 9 * capacity))) != HP_OK) return fail(rc);
    if ((rc = cuda_fail(cudaMalloc(&b->d_ctls, sizeof(hp::DevCtl*) * capacity))) != HP_OK) return fail(rc);
    if ((rc = cuda_fail(cudaMallocHost(&b->h_ctls, sizeof(hp::DevCtl*) * capacity))) != HP_OK) return fail(rc);
    if ((rc = cuda_fail(cudaMalloc(&b->d_counters, sizeof(int) * kLaunches))) != HP_OK) return fail(rc);
    if ((rc = cuda_fail(cudaMalloc(&b->d_plans, plans))) != HP_OK) return fail(rc);
    if ((rc = cuda_fail(cudaMallocHost(&b->h_plans, plans))) != HP_OK) return fail(rc);
    if ((rc = cuda_fail(cudaMalloc(&b->d_status, sizeof(unsigned) * capacity))) != HP_OK) return fail(rc);
    if ((rc = cuda_fail(cudaMallocHost(&b->h_status, sizeof(unsigned) * capacity))) != HP_OK) return fail(rc);
    for (int r = 0; r < kRing; ++r)
        if ((rc = cuda_fail(cudaEventCreateWithFlags(&b->ring_ev[r], cudaEventDisableTiming))) != HP_OK)
            return fail(rc);
    *out = b;
    return HP_OK;
}

int hp_batch_destroy(hp_batch* b) {
    if (!b) return HP_OK;
    cudaSetDevice(b->dev);
    if (b->stream) cudaStreamSynchronize(b->stream);
    drop_graphs(b);
    for (int r = 0; r < kRing; ++r)
        if (b->ring_ev[r]) cudaEventDestroy(b->ring_ev[r]);
    cudaFree(b->d_args);
    if (b->h_args) cudaFreeHost(b->h_args);
    cudaFree(b->d_ctls);
    if (b->h_ctls) cudaFreeHost(b->h_ctls);
    cudaFree(b->d_counters);
    cudaFree(b->d_plans);
    if (b->h_plans) cudaFreeHost(b->h_plans);
    cudaFree(b->d_status);
    if (b->h_status) cudaFreeHost(b->h_status);
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
    return HP_OK;
}

int hp_batch_add(hp_batch* b, hp_ctx* x) {
    if (!b || !x) return HP_ERR_ARG;
    if (x->dev != b->dev || x->prm.precision != b->precision) return HP_ERR_ARG;
    if ((int)b->members.size() >= b->cap) return HP_ERR_ARG;
    if (!x->attached) return HP_ERR_NOT_ATTACHED;
    if (x->box.g[0]) return HP_ERR_ARG;  // the batched sweeps carry no gravity source
    if (x->slab) return HP_ERR_ARG;      // nor the halos of a z slab
    if (x->box.pencil) return HP_ERR_ARG;  // nor the full-pencil solver
    if (std::find(b->members.begin(), b->members.end(), x) != b->members.end()) return HP_ERR_ARG;
    HP_CUDA(cudaSetDevice(b->dev));
    HP_CUDA(cudaStreamSynchronize(x->stream));  // the member's own work is finished
    b->members.push_back(x);
    b->tables_valid = false;
    return HP_OK;
}

int hp_batch_remove(hp_batch* b, hp_ctx* x) {
    if (!b || !x) return HP_ERR_ARG;
    auto it = std::find(b->members.begin(), b->members.end(), x);
    if (it == b->members.end()) return HP_ERR_ARG;
    HP_CUDA(cudaSetDevice(b->dev));
    HP_CUDA(cudaStreamSynchronize(b->stream));
    b->members.erase(it);
    b->tables_valid = false;
    return HP_OK;
}

int hp_batch_size(hp_batch* b) { return b ? (int)b->members.size() : 0; }

hp_ctx* hp_batch_member(hp_batch* b, int i) {
    if (!b || i < 0 || i >= (int)b->members.size()) return nullptr;
    return b->members[i];
}

int hp_batch_step(hp_batch* b, int nsteps, int use_graph) {
    if (!b || nsteps < 0) return HP_ERR_ARG;
    HP_CUDA(cudaSetDevice(b->dev));
    const int n = (int)b->members.size();
    if (n == 0) return HP_OK;
    std::vector<int> nrot(n);
    Plan dyn;
    for (int it = 0; it < nsteps; ++it) {
        hp::TraceRange tr("hp batch step");
        int rc = ensure_tables(b);
        if (rc != HP_OK) return rc;
        bool aligned = true;
        for (int m = 0; m < n; ++m) {
            nrot[m] = hp::nrot_of_step(b->members[m]->nstep_host);
            aligned = aligned && nrot[m] == nrot[0];
        }
        if (aligned) {
            const int r = nrot[0];
            const int* dplan = b->d_plans + (size_t)(kRing + r - 1) * b->plan_ints;
            if (use_graph) {
                cudaGraphExec_t& g = b->graph[r - 1];
                if (!g) {
                    cudaGraph_t graph;
                    HP_CUDA(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
                    const int k = enqueue_plan(b, b->static_plan[r - 1], dplan);
                    const cudaError_t ce = cudaStreamEndCapture(b->stream, &graph);
                    if (k < 0) {
                        if (ce == cudaSuccess) cudaGraphDestroy(graph);
                        return k;
                    }
                    HP_CUDA(ce);
                    const cudaError_t ie = cudaGraphInstantiate(&g, graph, 0);
                    cudaGraphDestroy(graph);
                    HP_CUDA(ie);
                    b->graph_kernels[r - 1] = k;
                }
                HP_CUDA(cudaGraphLaunch(g, b->stream));
                b->launches += b->graph_kernels[r - 1];
            } else {
                const int k = enqueue_plan(b, b->static_plan[r - 1], dplan);
                if (k < 0) return k;
                b->launches += k;
            }
        } else {
            build_plan(b, nrot, dyn);
            const int r = b->ring_next;
            b->ring_next = (r + 1) % kRing;
            HP_CUDA(cudaEventSynchronize(b->ring_ev[r]));  // the ring slot's previous copy has run
            int* h = b->h_plans + (size_t)r * b->plan_ints;
            int* d = b->d_plans + (size_t)r * b->plan_ints;
            memcpy(h, dyn.ints.data(), dyn.ints.size() * sizeof(int));
            HP_CUDA(cudaMemcpyAsync(d, h, dyn.ints.size() * sizeof(int), cudaMemcpyHostToDevice, b->stream));
            HP_CUDA(cudaEventRecord(b->ring_ev[r], b->stream));
            const int k = enqueue_plan(b, dyn, d);
            if (k < 0) return k;
            b->launches += k;
        }
        for (int m = 0; m < n; ++m) {
            b->members[m]->sweep_count += 3;
            b->members[m]->nstep_host += 1;
        }
    }
    return HP_OK;
}

int hp_batch_synchronize(hp_batch* b, int* status) {
    if (!b) return HP_ERR_ARG;
    HP_CUDA(cudaSetDevice(b->dev));
    const int n = (int)b->members.size();
    if (n == 0) {
        HP_CUDA(cudaStreamSynchronize(b->stream));
        return HP_OK;
    }
    int rc = ensure_tables(b);  // the control-block list of the current members
    if (rc != HP_OK) return rc;
    if (hp::launch_status_gather(b->d_ctls, n, b->d_status, b->stream) < 0) return HP_ERR_CUDA;
    b->launches += 1;
    HP_CUDA(cudaMemcpyAsync(b->h_status, b->d_status, sizeof(unsigned) * n, cudaMemcpyDeviceToHost, b->stream));
    HP_CUDA(cudaStreamSynchronize(b->stream));
    int first = HP_OK;
    for (int m = 0; m < n; ++m) {
        const int e = hp::status_error(b->h_status[m]);
        if (status) status[m] = e;
        if (first == HP_OK) first = e;
    }
    return first;
}

int hp_batch_set_tiles(hp_batch* b, int tile_x, int tile_y, int tile_z) {
    if (!b) return HP_ERR_ARG;
    const int t[3] = {tile_x, tile_y, tile_z};
    for (int a = 0; a < 3; ++a)  // the batched kernel runs the classic tiles
        if (t[a] < 0 || t[a] >= hp::kNumClassicTiles) return HP_ERR_ARG;
    HP_CUDA(cudaSetDevice(b->dev));
    HP_CUDA(cudaStreamSynchronize(b->stream));
    for (int a = 0; a < 3; ++a) b->tile[a] = t[a];
    b->tables_valid = false;
    return HP_OK;
}

int hp_batch_get_tiles(hp_batch* b, int* tiles) {
    if (!b || !tiles) return HP_ERR_ARG;
    for (int a = 0; a < 3; ++a) tiles[a] = b->tile[a];
    return HP_OK;
}

int hp_batch_autotune(hp_batch* b, int reps) {
    if (!b || reps < 1) return HP_ERR_ARG;
    const int n = (int)b->members.size();
    if (n == 0) return HP_OK;
    HP_CUDA(cudaSetDevice(b->dev));
    int rc = ensure_tables(b);
    if (rc != HP_OK) return rc;
    // scratch copies of every member's fields and control block
    size_t cells = 0;
    std::vector<size_t> off(n);
    for (int m = 0; m < n; ++m) {
        off[m] = cells;
        const hp::Box& x = b->members[m]->box;
        cells += (size_t)x.nx * x.ny * x.nz;
    }
    double* fields = nullptr;
    hp::DevCtl* sctl = nullptr;
    hp::SweepArgs* sargs = nullptr;
    hp::SweepArgs* hargs = nullptr;
    int* splan = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    std::vector<int> plan;
    float best[3] = {1e30f, 1e30f, 1e30f};
    int pick[3] = {b->tile[0], b->tile[1], b->tile[2]};
    rc = cuda_fail(cudaMalloc(&fields, cells * 5 * sizeof(double)));
    if (rc == HP_OK) rc = cuda_fail(cudaMalloc(&sctl, sizeof(hp::DevCtl) * n));
    if (rc == HP_OK) rc = cuda_fail(cudaMalloc(&sargs, sizeof(hp::SweepArgs) * 3 * n));
    if (rc == HP_OK) rc = cuda_fail(cudaMallocHost(&hargs, sizeof(hp::SweepArgs) * 3 * n));
    if (rc == HP_OK) rc = cuda_fail(cudaMalloc(&splan, sizeof(int) * (2 * n + 1)));
    if (rc == HP_OK) rc = cuda_fail(cudaEventCreate(&e0));
    if (rc == HP_OK) rc = cuda_fail(cudaEventCreate(&e1));
    if (rc == HP_OK) {
        for (int m = 0; m < n; ++m) {
            hp::Box sb = b->members[m]->box;
            const size_t nc = (size_t)sb.nx * sb.ny * sb.nz;
            for (int q = 0; q < 5; ++q) sb.f[q] = fields + 5 * off[m] + q * nc;
            for (int q = 0; q < 4; ++q) sb.snap[q] = nullptr;
            sb.ctl = sctl + m;
            for (int axis = 0; axis < 3; ++axis) hargs[m * 3 + axis] = hp::make_sweep_args(sb, axis, b->base[m], 0);
        }
        rc = cuda_fail(cudaMemcpyAsync(sargs, hargs, sizeof(hp::SweepArgs) * 3 * n, cudaMemcpyHostToDevice,
                                       b->stream));
    }
    for (int axis = 0; axis < 3 && rc == HP_OK; ++axis) {
        for (int tile = 0; tile < hp::kNumClassicTiles && rc == HP_OK; ++tile) {
            const int P_ = hp::kTilePencils[axis][tile];
            plan.assign(2 * n + 1, 0);
            int first = 0;
            for (int m = 0; m < n; ++m) {
                const hp::Box& x = b->members[m]->box;
                const long long np = axis == 0 ? (long long)x.ny * x.nz
                                               : (axis == 1 ? (long long)x.nx * x.nz : (long long)x.nx * x.ny);
                plan[m] = m * 3 + axis;
                plan[n + m] = first;
                first += (int)((np + P_ - 1) / P_);
            }
            plan[2 * n] = first;
            rc = cuda_fail(cudaStreamSynchronize(b->stream));  // the pageable plan copy below is then ordered
            if (rc == HP_OK)
                rc = cuda_fail(cudaMemcpy(splan, plan.data(), sizeof(int) * (2 * n + 1), cudaMemcpyHostToDevice));
            for (int m = 0; m < n && rc == HP_OK; ++m) {
                const hp::Box& x = b->members[m]->box;
                const size_t nc = (size_t)x.nx * x.ny * x.nz;
                for (int q = 0; q < 5 && rc == HP_OK; ++q)
                    rc = cuda_fail(cudaMemcpyAsync(fields + 5 * off[m] + q * nc, x.f[q], nc * sizeof(double),
                                                   cudaMemcpyDeviceToDevice, b->stream));
                if (rc == HP_OK)
                    rc = cuda_fail(cudaMemcpyAsync(sctl + m, x.ctl, sizeof(hp::DevCtl), cudaMemcpyDeviceToDevice,
                                                   b->stream));
            }
            hp::BatchLaunch bl;
            bl.args = sargs;
            bl.ent = splan;
            bl.nent = n;
            bl.nitems = first;
            bl.counter = b->d_counters;
            // warm-up launch, then reps timed launches (each a full sweep of every member)
            for (int r = 0; r <= reps && rc == HP_OK; ++r) {
                if (r == 1) rc = cuda_fail(cudaEventRecord(e0, b->stream));
                if (rc == HP_OK)
                    rc = cuda_fail(cudaMemsetAsync(b->d_counters, 0, sizeof(int), b->stream));
                if (rc == HP_OK && hp::launch_sweep_batch(bl, axis, tile, b->precision, b->stream) < 0)
                    rc = HP_ERR_CUDA;
                b->launches += 1;
            }
            if (rc == HP_OK) rc = cuda_fail(cudaEventRecord(e1, b->stream));
            if (rc == HP_OK) rc = cuda_fail(cudaEventSynchronize(e1));
            float ms = 0.f;
            if (rc == HP_OK) rc = cuda_fail(cudaEventElapsedTime(&ms, e0, e1));
            if (rc == HP_OK && ms < best[axis]) {
                best[axis] = ms;
                pick[axis] = tile;
            }
        }
    }
    cudaStreamSynchronize(b->stream);
    cudaFree(fields);
    cudaFree(sctl);
    cudaFree(sargs);
    if (hargs) cudaFreeHost(hargs);
    cudaFree(splan);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (rc != HP_OK) return rc;
    // the status words of the scratch sweeps went to the scratch blocks
    return hp_batch_set_tiles(b, pick[0], pick[1], pick[2]);
}

void* hp_batch_stream(hp_batch* b) { return b ? (void*)b->stream : nullptr; }

long long hp_batch_launch_count(hp_batch* b) { return b ? b->launches : 0; }

}  // extern "C"
