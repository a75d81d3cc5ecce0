// rpl_ensemble.cu -- the batching form: many independent FP32 models ("members") advanced together.
//
// Per RK3 stage one persistent launch of the ensemble kernel (rpl_tile32.cu) covers every member: its
// CTAs take (member, tile, tile shape) items from an atomic counter, so members of very different
// sizes fill the GPU together instead of one small grid at a time. One step (counter reset + three
// stage launches) is captured in a CUDA graph once and replayed. The tile shape of each size class
// comes from an autotuner that times the candidate shapes and keeps them in a text cache.
//
// Reference: none for the batching itself (time_step.jl:119-170 advances one model per call); each
// member's stage arithmetic is the single-model tile kernel's.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <fstream>
#include <map>
#include <new>
#include <sstream>
#include <string>
#include <vector>

#include "rpl_internal.h"

using rpl::Handle;
using rpl::TileArgs;

struct rpl_ensemble {
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    bool refract = false;
    bool use_graph = true;
    std::string cache;
    std::vector<Handle*> members;
    std::vector<double> dt;
    std::vector<int> shape;             // per member: index into kEnsembleShapes
    int64_t direct_cells = 0;           // members with at least this many cells take single-model launches
    std::vector<char> direct;           // per member: stages launched directly, not in the persistent kernel
    std::vector<std::string> key;       // per member: size-class key
    TileArgs* d_args = nullptr;         // [3][count]: stage-major
    int4* d_items = nullptr;
    size_t item_capacity = 0;
    int nitems = 0;
    unsigned int* d_counters = nullptr; // one per stage
    int grid = 0;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaEvent_t done = nullptr;
    cudaEvent_t ready = nullptr;
};

namespace {

int efail(int code, const std::string& msg) {
    rpl::set_last_error(msg);
    return code;
}

int ecuda(cudaError_t e, const char* what) {
    return efail(e == cudaErrorMemoryAllocation ? RPL_ERR_OOM : RPL_ERR_CUDA,
                 std::string(what) + ": " + cudaGetErrorString(e));
}

#define ENS_CUDA(call)                                   \
    do {                                                 \
        cudaError_t e_ = (call);                         \
        if (e_ != cudaSuccess) return ecuda(e_, #call);  \
    } while (0)

std::string class_key(const Handle& h, int device) {
    cudaDeviceProp prop{};
    cudaGetDeviceProperties(&prop, device);
    std::ostringstream s;
    s << "cc" << prop.major << prop.minor << "x" << prop.multiProcessorCount << " " << h.desc.Nx << " " << h.desc.Ny
      << " " << h.desc.Nk << " " << h.desc.Np << " " << h.desc.transport << " " << (h.d_cgmag ? 1 : 0);
    return s.str();
}

std::vector<int> candidates(int64_t Nk) {
    std::vector<int> c;
    const int L = rpl::tile_lanes(Nk);
    for (int v = 0; v < rpl::kNumEnsembleShapes; ++v)
        if (rpl::kEnsembleShapes[v].L == L) c.push_back(v);
    return c;
}

int default_shape(int64_t Nk) { return candidates(Nk).front(); }

int64_t tiles_of(const Handle& h, int v) {
    const rpl::TileShape& t = rpl::kEnsembleShapes[v];
    return ((h.desc.Nx + t.TX - 1) / t.TX) * ((h.desc.Ny + t.TY - 1) / t.TY);
}

void drop_graph(rpl_ensemble* e) {
    if (e->exec) cudaGraphExecDestroy(e->exec);
    if (e->graph) cudaGraphDestroy(e->graph);
    e->exec = nullptr;
    e->graph = nullptr;
}

// The stage arguments of every member, [stage][member].
int upload_args(rpl_ensemble* e) {
    const size_t M = e->members.size();
    std::vector<TileArgs> args(3 * M);
    for (size_t m = 0; m < M; ++m) {
        const Handle& h = *e->members[m];
        for (int s = 1; s <= 3; ++s) {
            const void* Nin = s == 1 ? h.N : (s == 2 ? h.A : h.B);
            void* Nout = s == 1 ? h.A : (s == 2 ? h.B : h.N);
            const rpl::StageParams p = rpl::make_params(h, e->dt[m], s);
            args[(s - 1) * M + m] = rpl::make_tile_args(h, p, Nin, h.N, Nout);
        }
    }
    ENS_CUDA(cudaMemcpyAsync(e->d_args, args.data(), args.size() * sizeof(TileArgs), cudaMemcpyHostToDevice,
                             e->stream));
    ENS_CUDA(cudaStreamSynchronize(e->stream));
    return RPL_OK;
}

// Work items (member, tile, shape) of the listed members, each with shape[m] (or `force_shape`).
// Members with the largest per-item work (more directions, then more kappa bins) come first, so the
// CTAs that finish early pick up the small items at the end.
int upload_items(rpl_ensemble* e, const std::vector<int>& which, int force_shape) {
    std::vector<int> order(which);
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
        const Handle& ha = *e->members[a];
        const Handle& hb = *e->members[b];
        if (ha.desc.Np != hb.desc.Np) return ha.desc.Np > hb.desc.Np;
        return ha.desc.Nk > hb.desc.Nk;
    });
    std::vector<int4> items;
    for (int m : order) {
        const int v = force_shape >= 0 ? force_shape : e->shape[m];
        const int64_t n = tiles_of(*e->members[m], v);
        for (int64_t t = 0; t < n; ++t) items.push_back(make_int4(m, (int)t, v, 0));
    }
    if (items.size() > (size_t)0x7fffffff) return efail(RPL_ERR_ARGUMENT, "ensemble has too many tiles");
    if (items.size() > e->item_capacity) {
        if (e->d_items) cudaFree(e->d_items);
        e->d_items = nullptr;
        ENS_CUDA(cudaMalloc((void**)&e->d_items, items.size() * sizeof(int4)));
        e->item_capacity = items.size();
    }
    if (!items.empty()) {
        ENS_CUDA(cudaMemcpyAsync(e->d_items, items.data(), items.size() * sizeof(int4), cudaMemcpyHostToDevice,
                                 e->stream));
        ENS_CUDA(cudaStreamSynchronize(e->stream));
    }
    e->nitems = (int)items.size();
    return RPL_OK;
}

// The persistent launches' items: every member that does not take direct launches.
int all_items(rpl_ensemble* e) {
    std::vector<int> all;
    for (size_t m = 0; m < e->members.size(); ++m)
        if (!e->direct[m]) all.push_back((int)m);
    drop_graph(e);
    return upload_items(e, all, -1);
}

// One RK3 step: per stage, the direct members' single-model stage launches (each fills the GPU on its
// own), then one persistent launch over the other members' tiles.
cudaError_t enqueue_step(rpl_ensemble* e) {
    const size_t M = e->members.size();
    cudaError_t err = cudaMemsetAsync(e->d_counters, 0, 3 * sizeof(unsigned int), e->stream);
    for (int s = 0; s < 3 && err == cudaSuccess; ++s) {
        for (size_t m = 0; m < M && err == cudaSuccess; ++m) {
            if (!e->direct[m]) continue;
            const Handle& h = *e->members[m];
            const void* Nin = s == 0 ? h.N : (s == 1 ? h.A : h.B);
            void* Nout = s == 0 ? h.A : (s == 1 ? h.B : h.N);
            err = rpl::launch_stage(h, rpl::make_params(h, e->dt[m], s + 1), Nin, h.N, Nout, e->stream);
        }
        if (err == cudaSuccess && e->nitems > 0)
            err = rpl::launch_ensemble_stage(e->refract, e->d_args + s * M, e->d_items, e->nitems,
                                             e->d_counters + s, e->grid, e->stream);
    }
    return err;
}

int capture_graph(rpl_ensemble* e) {
    drop_graph(e);
    ENS_CUDA(cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeThreadLocal));
    const cudaError_t err = enqueue_step(e);
    cudaGraph_t g = nullptr;
    const cudaError_t end = cudaStreamEndCapture(e->stream, &g);
    if (err != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        return ecuda(err, "ensemble step capture");
    }
    if (end != cudaSuccess) return ecuda(end, "cudaStreamEndCapture");
    e->graph = g;
    ENS_CUDA(cudaGraphInstantiate(&e->exec, e->graph, 0));
    return RPL_OK;
}

// Orders the ensemble stream after all members' pending work.
int join_members(rpl_ensemble* e) {
    for (Handle* h : e->members) {
        if (h->stream == e->stream) continue;
        ENS_CUDA(cudaEventRecord(e->ready, h->stream));
        ENS_CUDA(cudaStreamWaitEvent(e->stream, e->ready, 0));
    }
    return RPL_OK;
}

// Orders the members' streams after the ensemble stream's work.
int release_members(rpl_ensemble* e) {
    ENS_CUDA(cudaEventRecord(e->done, e->stream));
    for (Handle* h : e->members)
        if (h->stream != e->stream) ENS_CUDA(cudaStreamWaitEvent(h->stream, e->done, 0));
    return RPL_OK;
}

void advance_clocks(rpl_ensemble* e, int64_t nsteps) {
    for (size_t m = 0; m < e->members.size(); ++m) {
        for (int64_t k = 0; k < nsteps; ++k) e->members[m]->time += e->dt[m];
        e->members[m]->iteration += nsteps;
    }
}

std::map<std::string, int> read_cache(const std::string& path) {
    std::map<std::string, int> out;
    if (path.empty()) return out;
    std::ifstream f(path);
    std::string line;
    while (std::getline(f, line)) {
        // rpl-tile <key fields...> | <shape> <L> <TX> <TY> <microseconds>
        const size_t bar = line.find('|');
        if (line.rfind("rpl-tile ", 0) != 0 || bar == std::string::npos) continue;
        const std::string key = line.substr(9, bar - 10);
        std::istringstream r(line.substr(bar + 1));
        int v = -1, L = 0, TX = 0, TY = 0;
        if (!(r >> v >> L >> TX >> TY)) continue;
        if (v < 0 || v >= rpl::kNumEnsembleShapes) continue;
        const rpl::TileShape& t = rpl::kEnsembleShapes[v];
        if (t.L != L || t.TX != TX || t.TY != TY) continue;  // a cache from another build's shape table
        out[key] = v;
    }
    return out;
}

void append_cache(const std::string& path, const std::string& key, int v, double us) {
    if (path.empty()) return;
    std::ofstream f(path, std::ios::app);
    const rpl::TileShape& t = rpl::kEnsembleShapes[v];
    f << "rpl-tile " << key << " | " << v << " " << t.L << " " << t.TX << " " << t.TY << " " << us << "\n";
}

int check_ensemble(const rpl_ensemble* e) {
    if (!e) return efail(RPL_ERR_ARGUMENT, "null ensemble");
    cudaError_t err = cudaSetDevice(e->device);
    if (err != cudaSuccess) return ecuda(err, "cudaSetDevice");
    return RPL_OK;
}

void destroy(rpl_ensemble* e) {
    drop_graph(e);
    if (e->d_args) cudaFree(e->d_args);
    if (e->d_items) cudaFree(e->d_items);
    if (e->d_counters) cudaFree(e->d_counters);
    if (e->done) cudaEventDestroy(e->done);
    if (e->ready) cudaEventDestroy(e->ready);
    if (e->own_stream && e->stream) cudaStreamDestroy(e->stream);
    delete e;
}

}  // namespace

extern "C" {

int rpl_ensemble_autotune(rpl_ensemble* e, int32_t force) {
    int st = check_ensemble(e);
    if (st) return st;
    const std::map<std::string, int> cached = read_cache(e->cache);
    std::map<std::string, std::vector<int>> classes;
    // members with direct single-model launches never run in the persistent kernel: nothing to tune
    for (size_t m = 0; m < e->members.size(); ++m)
        if (!e->direct[m]) classes[e->key[m]].push_back((int)m);
    cudaEvent_t t0, t1;
    ENS_CUDA(cudaEventCreate(&t0));
    ENS_CUDA(cudaEventCreate(&t1));
    ENS_CUDA(cudaStreamSynchronize(e->stream));
    for (const auto& kv : classes) {
        const std::vector<int>& ms = kv.second;
        int best = -1;
        auto hit = cached.find(kv.first);
        if (!force && hit != cached.end()) best = hit->second;
        if (best < 0) {
            double best_us = INFINITY;
            for (int v : candidates(e->members[ms[0]]->desc.Nk)) {
                if ((st = upload_items(e, ms, v))) break;
                double t_min = INFINITY;
                for (int r = 0; r < 4; ++r) {  // one warm-up, three timed stage-1 launches
                    cudaError_t err = cudaMemsetAsync(e->d_counters, 0, sizeof(unsigned int), e->stream);
                    if (err == cudaSuccess) err = cudaEventRecord(t0, e->stream);
                    if (err == cudaSuccess)
                        err = rpl::launch_ensemble_stage(e->refract, e->d_args, e->d_items, e->nitems, e->d_counters,
                                                         e->grid, e->stream);
                    if (err == cudaSuccess) err = cudaEventRecord(t1, e->stream);
                    if (err == cudaSuccess) err = cudaEventSynchronize(t1);
                    float ms_ = 0.f;
                    if (err == cudaSuccess) err = cudaEventElapsedTime(&ms_, t0, t1);
                    if (err != cudaSuccess) {
                        st = ecuda(err, "autotune launch");
                        break;
                    }
                    if (r > 0) t_min = std::min(t_min, 1e3 * (double)ms_);
                }
                if (st) break;
                if (t_min < best_us) {
                    best_us = t_min;
                    best = v;
                }
            }
            if (st) break;
            append_cache(e->cache, kv.first, best, best_us);
        }
        for (int m : ms) e->shape[m] = best;
    }
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    if (st) {
        all_items(e);  // back to the full item list with the shapes chosen so far
        return st;
    }
    // the timing launches only wrote the members' stage-1 scratch buffers and error words
    for (Handle* h : e->members) ENS_CUDA(cudaMemsetAsync(h->d_err, 0, sizeof(unsigned int), e->stream));
    return all_items(e);
}

int rpl_ensemble_create(rpl_handle* const* members, const double* dt, int32_t count,
                        const rpl_ensemble_options* options, rpl_ensemble** out) {
    if (!out) return efail(RPL_ERR_ARGUMENT, "out must not be NULL");
    *out = nullptr;
    if (!members || !dt || count < 1) return efail(RPL_ERR_ARGUMENT, "need at least one member and its dt");
    if (options && options->abi_version != RPL_ABI_VERSION)
        return efail(RPL_ERR_ARGUMENT, "rpl_ensemble_options.abi_version does not match the library");
    std::vector<Handle*> hs(count);
    for (int i = 0; i < count; ++i) {
        if (!members[i]) return efail(RPL_ERR_ARGUMENT, "member " + std::to_string(i) + " is NULL");
        hs[i] = reinterpret_cast<Handle*>(members[i]);
        if (!(dt[i] > 0.0) || !std::isfinite(dt[i]))
            return efail(RPL_ERR_DT, "member " + std::to_string(i) + ": time step must be positive");
        for (int j = 0; j < i; ++j)
            if (hs[j] == hs[i]) return efail(RPL_ERR_ARGUMENT, "a model appears twice in the ensemble");
    }
    const Handle& h0 = *hs[0];
    for (int i = 0; i < count; ++i) {
        const Handle& h = *hs[i];
        const std::string who = "member " + std::to_string(i) + ": ";
        if (h.device != h0.device) return efail(RPL_ERR_ARGUMENT, who + "members must share one device");
        if (h.precision != RPL_FP32 || !rpl::tile32_supported(h))
            return efail(RPL_ERR_UNSUPPORTED,
                         who + "ensembles take FP32 models with 4 <= Nk <= 32, Nk % 4 == 0, Nx, Ny >= 3 and transport");
        if (h.desc.transport != h0.desc.transport)
            return efail(RPL_ERR_UNSUPPORTED, who + "members must share one transport kind");
        if (h.has_sources || h.n_terms) return efail(RPL_ERR_UNSUPPORTED, who + "ensemble members carry no sources");
        if (h.desc.transport == RPL_TRANSPORT_REFRACTION && !h.currents_set)
            return efail(RPL_ERR_STATE, who + "refraction transport needs rpl_set_currents first");
        if (h.pm)
            return efail(RPL_ERR_UNSUPPORTED, who + "ensemble members take prescribed currents, not pseudomomentum");
        if (h.smooth) return efail(RPL_ERR_UNSUPPORTED, who + "ensemble members carry no propagation smoothing");
    }
    cudaError_t err = cudaSetDevice(h0.device);
    if (err != cudaSuccess) return ecuda(err, "cudaSetDevice");
    rpl_ensemble* e = new (std::nothrow) rpl_ensemble();
    if (!e) return efail(RPL_ERR_OOM, "host allocation failed");
    e->device = h0.device;
    e->refract = h0.desc.transport == RPL_TRANSPORT_REFRACTION;
    e->use_graph = options ? options->use_graph != 0 : true;
    e->cache = (options && options->autotune_cache) ? options->autotune_cache : "";
    e->members = hs;
    e->dt.assign(dt, dt + count);
    e->direct_cells = options ? options->direct_cells : 0;
    if (e->direct_cells < 0) {
        destroy(e);
        return efail(RPL_ERR_ARGUMENT, "direct_cells must be >= 0");
    }
    for (int i = 0; i < count; ++i)
        e->direct.push_back(e->direct_cells > 0 && hs[i]->cells >= e->direct_cells ? 1 : 0);
    const std::map<std::string, int> cached = read_cache(e->cache);
    for (int i = 0; i < count; ++i) {
        e->key.push_back(class_key(*hs[i], e->device));
        auto hit = cached.find(e->key.back());
        e->shape.push_back(hit != cached.end() ? hit->second : default_shape(hs[i]->desc.Nk));
    }
    int st = RPL_OK;
    auto bail = [&](int code) {
        destroy(e);
        return code;
    };
    if ((err = cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking)) != cudaSuccess)
        return bail(ecuda(err, "cudaStreamCreate"));
    e->own_stream = true;
    if ((err = cudaEventCreateWithFlags(&e->done, cudaEventDisableTiming)) != cudaSuccess ||
        (err = cudaEventCreateWithFlags(&e->ready, cudaEventDisableTiming)) != cudaSuccess)
        return bail(ecuda(err, "cudaEventCreate"));
    if ((err = rpl::prepare_ensemble_kernels()) != cudaSuccess) return bail(ecuda(err, "ensemble kernel attributes"));
    e->grid = rpl::ensemble_grid(e->refract, e->device);
    if ((err = cudaMalloc((void**)&e->d_args, 3 * (size_t)count * sizeof(TileArgs))) != cudaSuccess)
        return bail(ecuda(err, "cudaMalloc"));
    if ((err = cudaMalloc((void**)&e->d_counters, 3 * sizeof(unsigned int))) != cudaSuccess)
        return bail(ecuda(err, "cudaMalloc"));
    if ((st = join_members(e))) return bail(st);
    if ((st = upload_args(e))) return bail(st);
    if (options && options->autotune) {
        if ((st = rpl_ensemble_autotune(e, 0))) return bail(st);
    } else if ((st = all_items(e))) {
        return bail(st);
    }
    *out = e;
    return RPL_OK;
}

int rpl_ensemble_destroy(rpl_ensemble* e) {
    if (!e) return RPL_OK;
    cudaSetDevice(e->device);
    if (e->stream) cudaStreamSynchronize(e->stream);
    destroy(e);
    return RPL_OK;
}

int rpl_ensemble_step_async(rpl_ensemble* e, int64_t nsteps) {
    int st = check_ensemble(e);
    if (st) return st;
    if (nsteps < 0) return efail(RPL_ERR_ARGUMENT, "nsteps must be non-negative");
    if (nsteps == 0) return RPL_OK;
    if ((st = join_members(e))) return st;
    if (e->use_graph && !e->exec && (st = capture_graph(e))) return st;
    for (int64_t k = 0; k < nsteps; ++k) {
        if (e->use_graph) ENS_CUDA(cudaGraphLaunch(e->exec, e->stream));
        else ENS_CUDA(enqueue_step(e));
    }
    advance_clocks(e, nsteps);
    return release_members(e);
}

int rpl_ensemble_step_sequential_async(rpl_ensemble* e, int64_t nsteps) {
    int st = check_ensemble(e);
    if (st) return st;
    if (nsteps < 0) return efail(RPL_ERR_ARGUMENT, "nsteps must be non-negative");
    if ((st = join_members(e))) return st;
    for (int64_t k = 0; k < nsteps; ++k)
        for (size_t m = 0; m < e->members.size(); ++m) {
            const Handle& h = *e->members[m];
            for (int s = 1; s <= 3; ++s) {
                const void* Nin = s == 1 ? h.N : (s == 2 ? h.A : h.B);
                void* Nout = s == 1 ? h.A : (s == 2 ? h.B : h.N);
                const rpl::StageParams p = rpl::make_params(h, e->dt[m], s);
                ENS_CUDA(rpl::launch_stage(h, p, Nin, h.N, Nout, e->stream));
            }
        }
    advance_clocks(e, nsteps);
    return release_members(e);
}

int rpl_ensemble_sync(rpl_ensemble* e) {
    int st = check_ensemble(e);
    if (st) return st;
    ENS_CUDA(cudaStreamSynchronize(e->stream));
    for (size_t m = 0; m < e->members.size(); ++m) {
        Handle* h = e->members[m];
        ENS_CUDA(cudaMemcpyAsync(h->h_err, h->d_err, sizeof(unsigned int), cudaMemcpyDeviceToHost, e->stream));
        ENS_CUDA(cudaStreamSynchronize(e->stream));
        if (*h->h_err) {
            ENS_CUDA(cudaMemsetAsync(h->d_err, 0, sizeof(unsigned int), e->stream));
            ENS_CUDA(cudaStreamSynchronize(e->stream));
            return efail(RPL_ERR_DEVICE, "member " + std::to_string(m) +
                                             ": a stage kernel produced non-finite wave action (time step too large?)");
        }
    }
    return RPL_OK;
}

int rpl_ensemble_step(rpl_ensemble* e, int64_t nsteps) {
    int st = rpl_ensemble_step_async(e, nsteps);
    if (st) return st;
    return rpl_ensemble_sync(e);
}

int rpl_ensemble_shape(const rpl_ensemble* e, int32_t member, int32_t* lanes, int32_t* tile_x, int32_t* tile_y) {
    if (!e) return efail(RPL_ERR_ARGUMENT, "null ensemble");
    if (member < 0 || member >= (int32_t)e->members.size()) return efail(RPL_ERR_ARGUMENT, "member out of range");
    const rpl::TileShape& t = rpl::kEnsembleShapes[e->shape[member]];
    if (lanes) *lanes = t.L;
    if (tile_x) *tile_x = t.TX;
    if (tile_y) *tile_y = t.TY;
    return RPL_OK;
}

int rpl_ensemble_set_stream(rpl_ensemble* e, void* stream) {
    int st = check_ensemble(e);
    if (st) return st;
    ENS_CUDA(cudaStreamSynchronize(e->stream));
    drop_graph(e);
    if (e->own_stream) cudaStreamDestroy(e->stream);
    e->own_stream = false;
    e->stream = (cudaStream_t)stream;
    if (!e->stream) {  // NULL: back to a stream of the ensemble's own (graphs cannot capture the legacy stream)
        ENS_CUDA(cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking));
        e->own_stream = true;
    }
    return RPL_OK;
}

}  // extern "C"
