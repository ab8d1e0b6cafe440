// Batch of many resident lattices advanced together (C ABI wake_batch_* in
// include/wake_gpu.h). No reference counterpart: the reference steps one
// LatticeGrid per object and call (src/grid/lattice_grid_2d.cpp:195-265); a
// parameter sweep or a serving loop runs one such object per job. Here every
// member keeps its own state, geometry, parameters and force history (it is an
// ordinary wake_grid), and one step of the whole batch is three launches:
//
//   bulk launch    : every pure-gather row of every member (k_step_fast_batch)
//   general launch : every other row (k_step_batch), on a forked stream
//   reduction      : one block per member with momentum exchange
//
// Each launch reads the member's step arguments from a device table, so members
// of any size share a launch and the per-node arithmetic is the single-lattice
// arithmetic: a member's results do not depend on what else is in the batch.
#include <chrono>
#include <cstring>
#include <string>
#include <vector>

#include "engine.cuh"

namespace wk {

struct MemRed {  // one member's momentum-exchange reduction
    const double* contrib;
    int n;
    unsigned* hist_step;
    double* hist;
    int hist_cap;
};

__global__ void __launch_bounds__(256) k_batch_mem_reduce(const MemRed* __restrict__ list) {
    const MemRed m = list[blockIdx.x];
    mem_reduce_block(m.contrib, m.n, m.hist_step, m.hist, m.hist_cap);
}

}  // namespace wk

using namespace wk;

struct wake_batch {
    struct Member {
        wake_grid* g;
        cudaStream_t saved_stream;  // the member's stream before it joined
    };
    int Q = 0, storage = 0;
    std::vector<Member> members;
    cudaStream_t stream = nullptr, side = nullptr;
    bool own_stream = false;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;

    DevMem d_dom, d_fast, d_gen, d_red;
    std::vector<BatchDom> up_dom;  // table as last uploaded
    std::vector<MemRed> up_red;
    int n_fast = 0, n_gen = 0, n_red = 0;
    bool idx32 = true;
    bool tiles = false;      // one persistent tile launch per step (k_step_tiles)
    int kernel_variant = 0;  // 0 automatic, 1 direct, 2 persistent tiles (when every member allows it)
    DevMem d_tiles, d_gen4, d_mixed;  // tiles, general segments with entries, spans outside the tiles
    int n_tiles = 0, n_tile_gen = 0, n_mixed = 0;
    int coll = 0, les = 0;
    int parity = 0;  // batch steps taken, mod 2

    // row lists are rebuilt when the members or any member's geometry change
    std::vector<std::pair<const wake_grid*, unsigned long long>> layout;
    std::vector<int> gen_first;
    unsigned shape = 0;  // bumped when launch shapes or table addresses change
    // host seconds spent in wake_batch_step: preparing members and tables, capturing and
    // instantiating graphs, issuing launches (a launch that waits for queue space counts here)
    double host_s[3] = {0.0, 0.0, 0.0};

    int tpb_fast = 64, tpb_gen = 128;

    cudaGraphExec_t graph = nullptr;
    int graph_steps = 0, graph_parity = -1;
    unsigned graph_shape = ~0u;

    ~wake_batch() {
        if (stream && cudaStreamSynchronize(stream) == cudaSuccess && (!side || cudaStreamSynchronize(side) == cudaSuccess)) {
            d_dom.release();
            d_fast.release();
            d_gen.release();
            d_red.release();
            d_tiles.release();
            d_gen4.release();
            d_mixed.release();
        }
        if (graph) cudaGraphExecDestroy(graph);
        if (own_stream && stream) cudaStreamDestroy(stream);
        if (side) cudaStreamDestroy(side);
        if (ev_fork) cudaEventDestroy(ev_fork);
        if (ev_join) cudaEventDestroy(ev_join);
    }
    void drop_graph() {
        if (graph) cudaGraphExecDestroy(graph);
        graph = nullptr;
        graph_shape = ~0u;
    }
};

namespace {

bool valid_batch(wake_batch* b) {
    if (!b) {
        set_error(WAKE_ERR_INVALID, "null wake_batch handle");
        return false;
    }
    return true;
}

// Rebuild the concatenated row lists when the membership or a member's geometry changed.
int build_rows(wake_batch* b) {
    std::vector<std::pair<const wake_grid*, unsigned long long>> layout;
    layout.reserve(b->members.size());
    for (const auto& m : b->members) layout.emplace_back(m.g, m.g->geom_version);
    if (layout == b->layout && b->gen_first.size() == b->members.size()) return WAKE_OK;
    // queued steps may still read the old lists: let them finish, then lists can move freely
    WK_CUDA(cudaStreamSynchronize(b->stream));
    if (b->side) WK_CUDA(cudaStreamSynchronize(b->side));
    std::vector<uint4> fast, tiles, gen4, mixed;
    std::vector<uint2> gen;
    b->gen_first.assign(b->members.size(), 0);
    for (std::size_t i = 0; i < b->members.size(); ++i) {
        const wake_grid* g = b->members[i].g;
        const unsigned m = static_cast<unsigned>(i);
        for (uint4 sp : g->h_fast_rows) fast.push_back(make_uint4(m, sp.y, sp.z, sp.w));
        b->gen_first[i] = static_cast<int>(gen.size());
        for (unsigned r : g->h_gen_rows) gen.push_back(make_uint2(m, r));
        for (uint4 t : g->h_tiles) tiles.push_back(make_uint4(m, t.y, t.z, 0u));
        for (uint4 t : g->h_gen4) gen4.push_back(make_uint4(m, t.y, t.z, 0u));
        for (uint4 sp : g->h_mixed) mixed.push_back(make_uint4(m, sp.y, sp.z, sp.w));
    }
    WK_CUDA(b->d_mixed.grow(sizeof(uint4) * std::max<std::size_t>(1, mixed.size())));
    if (!mixed.empty())
        WK_CUDA(cudaMemcpyAsync(b->d_mixed.p, mixed.data(), sizeof(uint4) * mixed.size(), cudaMemcpyHostToDevice,
                                b->stream));
    b->n_mixed = static_cast<int>(mixed.size());
    WK_CUDA(b->d_tiles.grow(sizeof(uint4) * std::max<std::size_t>(1, tiles.size())));
    WK_CUDA(b->d_gen4.grow(sizeof(uint4) * std::max<std::size_t>(1, gen4.size())));
    if (!tiles.empty())
        WK_CUDA(cudaMemcpyAsync(b->d_tiles.p, tiles.data(), sizeof(uint4) * tiles.size(), cudaMemcpyHostToDevice,
                                b->stream));
    if (!gen4.empty())
        WK_CUDA(cudaMemcpyAsync(b->d_gen4.p, gen4.data(), sizeof(uint4) * gen4.size(), cudaMemcpyHostToDevice,
                                b->stream));
    b->n_tiles = static_cast<int>(tiles.size());
    b->n_tile_gen = static_cast<int>(gen4.size());
    WK_CUDA(b->d_fast.grow(sizeof(uint4) * std::max<std::size_t>(1, fast.size())));
    WK_CUDA(b->d_gen.grow(sizeof(uint2) * std::max<std::size_t>(1, gen.size())));
    if (!fast.empty())
        WK_CUDA(cudaMemcpyAsync(b->d_fast.p, fast.data(), sizeof(uint4) * fast.size(), cudaMemcpyHostToDevice, b->stream));
    if (!gen.empty())
        WK_CUDA(cudaMemcpyAsync(b->d_gen.p, gen.data(), sizeof(uint2) * gen.size(), cudaMemcpyHostToDevice, b->stream));
    WK_CUDA(cudaStreamSynchronize(b->stream));  // the host vectors go out of scope
    b->n_fast = static_cast<int>(fast.size());
    b->n_gen = static_cast<int>(gen.size());
    b->layout = std::move(layout);
    b->up_dom.clear();  // force a table upload
    ++b->shape;
    return WAKE_OK;
}

// Step-argument table and reduction list of the current members; uploaded when changed.
int build_tables(wake_batch* b) {
    const std::size_t n = b->members.size();
    std::vector<BatchDom> dom(n);
    std::vector<MemRed> red;
    b->idx32 = true;
    bool tiles = b->kernel_variant == 2 && n > 0;
    for (std::size_t i = 0; i < n; ++i) {
        wake_grid* g = b->members[i].g;
        tiles = tiles && tile_row_ok(g->nx, static_cast<int>(g->elem));
        BatchDom d;
        std::memset(&d, 0, sizeof d);
        d.a = grid_step_args(g);
        d.buf[0] = g->A.p;
        d.buf[1] = g->B.p;
        d.tbuf[0] = g->tbuf(0);
        d.tbuf[1] = g->tbuf(1);
        d.cur0 = g->cur ^ b->parity;
        d.gen_first = b->gen_first[i];
        dom[i] = d;
        if (static_cast<long long>(g->Q) * g->pitch >= (1ll << 32)) b->idx32 = false;
        if (g->mem_on) {
            MemRed m;
            std::memset(&m, 0, sizeof m);
            m.contrib = d.a.mem.contrib;
            m.n = d.a.mem.n_nodes;
            m.hist_step = d.a.mem.hist_step;
            m.hist = d.a.mem.hist;
            m.hist_cap = d.a.mem.hist_cap;
            red.push_back(m);
        }
    }
    if (tiles != b->tiles) {
        b->tiles = tiles;
        ++b->shape;  // a captured graph holds the other kernel
    }
    const bool same_dom = dom.size() == b->up_dom.size() &&
                          (dom.empty() || std::memcmp(dom.data(), b->up_dom.data(), sizeof(BatchDom) * n) == 0);
    const bool same_red = red.size() == b->up_red.size() &&
                          (red.empty() || std::memcmp(red.data(), b->up_red.data(), sizeof(MemRed) * red.size()) == 0);
    if (same_dom && same_red) return WAKE_OK;
    WK_CUDA(cudaStreamSynchronize(b->stream));  // queued steps may still read the old tables
    if (b->side) WK_CUDA(cudaStreamSynchronize(b->side));
    const void* old_dom = b->d_dom.p;
    const void* old_red = b->d_red.p;
    const int old_nred = b->n_red;
    WK_CUDA(b->d_dom.grow(sizeof(BatchDom) * std::max<std::size_t>(1, n)));
    WK_CUDA(b->d_red.grow(sizeof(MemRed) * std::max<std::size_t>(1, red.size())));
    if (n) WK_CUDA(cudaMemcpyAsync(b->d_dom.p, dom.data(), sizeof(BatchDom) * n, cudaMemcpyHostToDevice, b->stream));
    if (!red.empty())
        WK_CUDA(cudaMemcpyAsync(b->d_red.p, red.data(), sizeof(MemRed) * red.size(), cudaMemcpyHostToDevice, b->stream));
    WK_CUDA(cudaStreamSynchronize(b->stream));
    b->n_red = static_cast<int>(red.size());
    b->up_dom = std::move(dom);
    b->up_red = std::move(red);
    // a captured graph keeps launch shapes and table addresses, not the table contents
    if (old_dom != b->d_dom.p || old_red != b->d_red.p || old_nred != b->n_red) ++b->shape;
    return WAKE_OK;
}

int batch_steps(wake_batch* b, int n) {
    if (b->tiles) {
        for (int s = 0; s < n; ++s) {
            const TileArgs t{b->d_tiles.as<uint4>(), b->n_tiles, b->d_gen4.as<uint4>(), b->n_tile_gen,
                             b->d_dom.as<BatchDom>(), b->parity, b->d_mixed.as<uint4>(), b->n_mixed};
            StepArgs unused{};
            WK_CUDA(launch_tiles_any(b->Q, b->coll, b->storage, b->les != 0, unused, t, b->stream));
            if (b->n_red > 0) {
                k_batch_mem_reduce<<<b->n_red, 256, 0, b->stream>>>(b->d_red.as<MemRed>());
                WK_CUDA(cudaGetLastError());
            }
            b->parity ^= 1;
        }
        return WAKE_OK;
    }
    for (int s = 0; s < n; ++s) {
        BatchArgs fa{b->d_dom.as<BatchDom>(), nullptr, 0, b->parity, b->d_fast.as<uint4>(), b->n_fast};
        BatchArgs ga{b->d_dom.as<BatchDom>(), b->d_gen.as<uint2>(), b->n_gen, b->parity, nullptr, 0};
        const bool fork = b->n_fast > 0 && (b->n_gen > 0 || b->n_red > 0);
        cudaStream_t side = fork ? b->side : b->stream;
        if (fork) {
            WK_CUDA(cudaEventRecord(b->ev_fork, b->stream));
            WK_CUDA(cudaStreamWaitEvent(b->side, b->ev_fork, 0));
        }
        WK_CUDA(launch_batch_any(b->Q, b->coll, b->storage, b->les != 0, ga, b->tpb_gen, side, false, b->idx32));
        if (b->n_red > 0) {
            k_batch_mem_reduce<<<b->n_red, 256, 0, side>>>(b->d_red.as<MemRed>());
            WK_CUDA(cudaGetLastError());
        }
        WK_CUDA(launch_batch_any(b->Q, b->coll, b->storage, b->les != 0, fa, b->tpb_fast, b->stream, true, b->idx32));
        if (fork) {
            WK_CUDA(cudaEventRecord(b->ev_join, b->side));
            WK_CUDA(cudaStreamWaitEvent(b->stream, b->ev_join, 0));
        }
        b->parity ^= 1;
    }
    return WAKE_OK;
}

// Prepare every member and the tables for the next steps.
int batch_prepare(wake_batch* b) {
    if (b->members.empty()) return WAKE_OK;
    const wake_grid* g0 = b->members[0].g;
    for (const auto& m : b->members) {
        if (m.g->collision != g0->collision || m.g->les != g0->les)
            return set_error(WAKE_ERR_INVALID, "wake_batch: members differ in collision model or LES switch");
    }
    b->coll = g0->collision;
    b->les = g0->les;
    for (const auto& m : b->members) {
        const int r = grid_prepare(m.g);
        if (r) return r;
    }
    int r = build_rows(b);
    if (r) return r;
    return build_tables(b);
}

}  // namespace

extern "C" {

wake_batch* wake_batch_create(int q, int storage) {
    if (!(q == 9 || q == 19 || q == 27) || storage < 0 || storage > 3) {
        set_error(WAKE_ERR_INVALID, "wake_batch_create: invalid lattice or storage");
        return nullptr;
    }
    auto* b = new wake_batch();
    b->Q = q;
    b->storage = storage;
    cudaError_t e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) b->own_stream = true;
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&b->side, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->ev_fork, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->ev_join, cudaEventDisableTiming);
    if (e != cudaSuccess) {
        set_error(WAKE_ERR_CUDA, std::string("wake_batch_create: ") + cudaGetErrorString(e));
        delete b;
        return nullptr;
    }
    return b;
}

void wake_batch_destroy(wake_batch* b) {
    if (!b) return;
    if (b->stream) cudaStreamSynchronize(b->stream);
    for (auto& m : b->members) wake_grid_set_stream(m.g, m.saved_stream);
    delete b;
}

int wake_batch_add(wake_batch* b, wake_grid* g) {
    if (!valid_batch(b) || !grid_valid(g)) return WAKE_ERR_INVALID;
    if (g->Q != b->Q || g->storage != b->storage)
        return set_error(WAKE_ERR_INVALID, "wake_batch_add: lattice or storage differs from the batch");
    for (const auto& m : b->members)
        if (m.g == g) return set_error(WAKE_ERR_INVALID, "wake_batch_add: grid is already a member");
    // the member's work (preparation, reads) is ordered on the batch stream from now on
    WK_CUDA(cudaStreamSynchronize(g->stream));
    const cudaStream_t saved = g->own_stream ? nullptr : g->stream;
    int r = wake_grid_set_stream(g, b->stream);
    if (r) return r;
    b->members.push_back({g, saved});
    return static_cast<int>(b->members.size()) - 1;
}

int wake_batch_remove(wake_batch* b, wake_grid* g) {
    if (!valid_batch(b) || !grid_valid(g)) return WAKE_ERR_INVALID;
    for (std::size_t i = 0; i < b->members.size(); ++i) {
        if (b->members[i].g != g) continue;
        WK_CUDA(cudaStreamSynchronize(b->stream));
        const cudaStream_t saved = b->members[i].saved_stream;
        b->members.erase(b->members.begin() + static_cast<long>(i));
        return wake_grid_set_stream(g, saved);
    }
    return set_error(WAKE_ERR_INVALID, "wake_batch_remove: grid is not a member");
}

int wake_batch_size(wake_batch* b) { return valid_batch(b) ? static_cast<int>(b->members.size()) : WAKE_ERR_INVALID; }

int wake_batch_set_stream(wake_batch* b, void* stream) {
    if (!valid_batch(b)) return WAKE_ERR_INVALID;
    WK_CUDA(cudaStreamSynchronize(b->stream));
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (!s) {
        if (!b->own_stream) {
            WK_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
            b->own_stream = true;
        } else {
            s = b->stream;
        }
    } else if (b->own_stream) {
        cudaStreamDestroy(b->stream);
        b->own_stream = false;
    }
    b->stream = s;
    for (auto& m : b->members) {
        const int r = wake_grid_set_stream(m.g, s);
        if (r) return r;
    }
    b->drop_graph();
    return WAKE_OK;
}

int wake_batch_use_graph(wake_batch* b, int steps_per_graph) {
    if (!valid_batch(b)) return WAKE_ERR_INVALID;
    if (steps_per_graph < 0) return set_error(WAKE_ERR_INVALID, "negative graph size");
    b->graph_steps = steps_per_graph > 0 && steps_per_graph % 2 ? steps_per_graph + 1 : steps_per_graph;
    b->drop_graph();
    return WAKE_OK;
}

int wake_batch_set_block(wake_batch* b, int threads_bulk, int threads_general) {
    if (!valid_batch(b)) return WAKE_ERR_INVALID;
    if (threads_bulk < 32 || threads_bulk > WK_FAST_MAX_THREADS || threads_bulk % 32 || threads_general < 32 ||
        threads_general > 512 || threads_general % 32)
        return set_error(WAKE_ERR_INVALID, "wake_batch_set_block: bulk 32..256 (at most the fast kernels' bound), "
                                           "general 32..512, multiples of 32");
    b->tpb_fast = threads_bulk;
    b->tpb_gen = threads_general;
    b->drop_graph();
    return WAKE_OK;
}

int wake_batch_get_block(wake_batch* b) { return valid_batch(b) ? b->tpb_fast : WAKE_ERR_INVALID; }

int wake_batch_set_kernel(wake_batch* b, int variant) {
    if (!valid_batch(b)) return WAKE_ERR_INVALID;
    if (variant < 0 || variant > 2) return set_error(WAKE_ERR_INVALID, "wake_batch_set_kernel: variant 0, 1 or 2");
    b->kernel_variant = variant;
    b->up_dom.clear();  // re-evaluated with the tables
    b->drop_graph();
    return WAKE_OK;
}

int wake_batch_step(wake_batch* b, int n) {
    if (!valid_batch(b)) return WAKE_ERR_INVALID;
    if (n < 0) return set_error(WAKE_ERR_INVALID, "negative step count");
    if (n == 0 || b->members.empty()) return WAKE_OK;
    using clock = std::chrono::steady_clock;
    auto t0 = clock::now();
    auto lap = [&](int phase) {
        const auto t = clock::now();
        b->host_s[phase] += std::chrono::duration<double>(t - t0).count();
        t0 = t;
    };
    int r = batch_prepare(b);
    lap(0);
    if (r) return r;
    int done = 0;
    const int gs = b->graph_steps;
    if (gs > 0 && n >= gs) {
        if (!b->graph || b->graph_shape != b->shape || b->graph_parity != b->parity) {
            b->drop_graph();
            const int p0 = b->parity;
            cudaGraph_t graph = nullptr;
            WK_CUDA(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
            r = batch_steps(b, gs);
            const cudaError_t e = cudaStreamEndCapture(b->stream, &graph);
            b->parity = p0;
            if (r) {
                if (graph) cudaGraphDestroy(graph);
                return r;
            }
            if (e != cudaSuccess) return set_error(WAKE_ERR_CUDA, std::string("batch graph capture: ") + cudaGetErrorString(e));
            const cudaError_t e2 = cudaGraphInstantiate(&b->graph, graph, 0);
            cudaGraphDestroy(graph);
            if (e2 != cudaSuccess) {
                b->graph = nullptr;
                return set_error(WAKE_ERR_CUDA, std::string("batch graph instantiate: ") + cudaGetErrorString(e2));
            }
            const cudaError_t e3 = cudaGraphUpload(b->graph, b->stream);
            if (e3 != cudaSuccess) return set_error(WAKE_ERR_CUDA, std::string("batch graph upload: ") + cudaGetErrorString(e3));
            b->graph_shape = b->shape;
            b->graph_parity = p0;
        }
        lap(1);
        while (n - done >= gs) {  // gs is even: the parity returns to graph_parity
            WK_CUDA(cudaGraphLaunch(b->graph, b->stream));
            done += gs;
        }
    }
    r = batch_steps(b, n - done);
    for (auto& m : b->members) grid_advanced(m.g, n);
    lap(2);
    return r;
}

int wake_batch_host_seconds(wake_batch* b, double* prepare_s, double* capture_s, double* launch_s) {
    if (!valid_batch(b)) return WAKE_ERR_INVALID;
    if (prepare_s) *prepare_s = b->host_s[0];
    if (capture_s) *capture_s = b->host_s[1];
    if (launch_s) *launch_s = b->host_s[2];
    return WAKE_OK;
}

int wake_batch_synchronize(wake_batch* b) {
    if (!valid_batch(b)) return WAKE_ERR_INVALID;
    WK_CUDA(cudaStreamSynchronize(b->stream));
    for (std::size_t i = 0; i < b->members.size(); ++i) {
        const int r = grid_check_status(b->members[i].g);
        if (r) return set_error(r, "wake_batch member " + std::to_string(i) + ": " + wake_gpu_last_error());
    }
    return WAKE_OK;
}

int wake_batch_info(wake_batch* b, long long* nodes, int* bulk_rows, int* general_rows, int* launches_per_step) {
    if (!valid_batch(b)) return WAKE_ERR_INVALID;
    const int r = batch_prepare(b);
    if (r) return r;
    long long nn = 0;
    for (const auto& m : b->members) nn += m.g->N;
    if (nodes) *nodes = nn;
    if (bulk_rows) *bulk_rows = b->n_fast;
    if (general_rows) *general_rows = b->n_gen;
    if (launches_per_step)
        *launches_per_step = b->tiles ? 1 + (b->n_red > 0) : (b->n_fast > 0) + (b->n_gen > 0) + (b->n_red > 0);
    return WAKE_OK;
}

// Time `steps` real steps for each bulk block size of {32, 64, 128, 256} within the
// kernels' launch bound (plain launches, CUDA events on the batch stream) and keep
// the fastest. The members advance `steps` per size tried; results do not depend on
// the block size.
int wake_batch_autotune(wake_batch* b, int steps, int* best_threads) {
    if (!valid_batch(b)) return WAKE_ERR_INVALID;
    if (steps < 1) return set_error(WAKE_ERR_INVALID, "wake_batch_autotune: steps must be positive");
    if (b->members.empty()) return WAKE_OK;
    int r = batch_prepare(b);
    if (r) return r;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    WK_CUDA(cudaEventCreate(&e0));
    if (cudaEventCreate(&e1) != cudaSuccess) {
        cudaEventDestroy(e0);
        return set_error(WAKE_ERR_CUDA, "wake_batch_autotune: event creation failed");
    }
    const int keep = b->tpb_fast;
    int best = keep;
    float best_ms = -1.f;
    for (int t : {32, 64, 128, 256}) {
        if (t > WK_FAST_MAX_THREADS) break;
        b->tpb_fast = t;
        cudaEventRecord(e0, b->stream);
        r = batch_steps(b, steps);
        cudaEventRecord(e1, b->stream);
        if (r) break;
        for (auto& m : b->members) grid_advanced(m.g, steps);
        float ms = 0.f;
        if (cudaEventSynchronize(e1) != cudaSuccess || cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess) {
            r = set_error(WAKE_ERR_CUDA, "wake_batch_autotune: timing failed");
            break;
        }
        if (best_ms < 0.f || ms < best_ms) {
            best_ms = ms;
            best = t;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    b->tpb_fast = r ? keep : best;
    b->drop_graph();
    if (best_threads) *best_threads = b->tpb_fast;
    return r;
}

}  // extern "C"
