// batch.cu -- many clouds reconstructed under one CUDA graph per iteration,
// with the grid sums of all clouds in one persistent launch.
#include "batch.cuh"

#include <algorithm>

namespace dwg {

Batch::~Batch() {
    if (s) cudaStreamSynchronize(s);
    if (graph_exec) cudaGraphExecDestroy(graph_exec);
    if (graph) cudaGraphDestroy(graph);
    {
        // each pipeline synchronises its own stream first, and the batch's
        // stream (its persistent launch reads every cloud) was drained above
        FreeScope idle(nullptr, true);
        clouds.clear();
    }
    for (cudaEvent_t e : ev_done)
        if (e) cudaEventDestroy(e);
    if (ev_fork) cudaEventDestroy(ev_fork);
    if (ev_mid) cudaEventDestroy(ev_mid);
    if (s) cudaStreamDestroy(s);
}

int Batch::join_in() {
    DWG_CHECK_CUDA(cudaEventRecord(ev_fork, caller));
    DWG_CHECK_CUDA(cudaStreamWaitEvent(s, ev_fork, 0));
    return DWG_OK;
}

int Batch::join_out() {
    DWG_CHECK_CUDA(cudaEventRecord(ev_fork, s));
    DWG_CHECK_CUDA(cudaStreamWaitEvent(caller, ev_fork, 0));
    return DWG_OK;
}

int Batch::setup(const float* const* points_dev, const int* counts, int n, const dwg_params* params,
                 cudaStream_t stream) {
    DWG_REQUIRE(points_dev && counts && params && n >= 1, "batch: need at least one cloud");
    for (int i = 0; i < n; ++i) {
        DWG_REQUIRE(params[i].in_normal == 3, "batch: cloud %d: only the Gauss-map start (in_normal 3)", i);
        DWG_REQUIRE(params[i].tile == params[0].tile && params[i].precision == params[0].precision,
                    "batch: cloud %d: tile and precision must be the same for every cloud", i);
    }
    caller = stream;
    DWG_CHECK_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    DWG_CHECK_CUDA(cudaEventCreateWithFlags(&ev_fork, cudaEventDisableTiming));
    DWG_CHECK_CUDA(cudaEventCreateWithFlags(&ev_mid, cudaEventDisableTiming));
    ev_done.assign((size_t)2 * n, nullptr);
    for (auto& e : ev_done) DWG_CHECK_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    DWG_TRY(join_in());
    clouds.reserve((size_t)n);
    for (int i = 0; i < n; ++i) {
        clouds.emplace_back(new dwg_pipeline());
        int st = clouds.back()->p.setup(points_dev[i], nullptr, counts[i], params[i], s);
        if (st != DWG_OK) {
            const std::string msg = dwg_last_error();
            set_error("batch: cloud %d: %s", i, msg.c_str());
            return st;
        }
    }
    // what the clouds' grid lists and weights may not take: room for the
    // workspaces that the first iteration sizes (marching cubes, kNN, repair)
    reserve = device_free_bytes() / 4;
    return join_out();
}

// Weight slots for the clouds' kept grid lists, then the grid sums of the
// clouds without lists as one work list.  Every listed cloud with weights
// wanted gets one slot (its most used sigma) in order of list size while
// they fit above the reserve, then a second, and so on: the weights save
// about the same time per byte in every cloud, the first slot the most.
int Batch::prepare_grid() {
    const int n = (int)clouds.size();
    std::vector<int> order;
    for (int i = 0; i < n; ++i) {
        const GwnList& L = clouds[i]->p.glist;
        if (clouds[i]->p.prm.grid_lists && L.valid && !L.too_big && L.wslots > 0 && L.wstate.ptr && L.entries)
            order.push_back(i);
    }
    std::sort(order.begin(), order.end(),
              [&](int a, int b) { return clouds[a]->p.glist.entries > clouds[b]->p.glist.entries; });
    std::vector<int> slots((size_t)n, 0);
    {
        // the first iteration has sized every workspace the graph uses; the
        // final pass runs after the lists are released (finalize), so a
        // small margin stays free
        const size_t keep = std::min(reserve, (size_t)4 << 30);
        const size_t fr = device_free_bytes();
        size_t room = fr > keep ? fr - keep : 0;
        for (int pass = 1; pass <= kGwnWeightSlots; ++pass)
            for (int i : order) {
                const GwnList& L = clouds[i]->p.glist;
                const size_t need = (size_t)L.entries * 32 * sizeof(float2);  // one grid slot
                if (L.wslots < pass || slots[i] != pass - 1 || need > room) continue;
                slots[i] = pass;
                room -= need;
            }
    }
    for (int i : order)
        if (slots[i] > 0 && gwn_list_add_weights(clouds[i]->p.glist, slots[i], clouds[i]->p.s) != DWG_OK) {
            cudaGetLastError();  // no room after all: this cloud replays its lists without weights
        }
    std::vector<GwnBatchItem> items;
    listed.assign((size_t)n, 0);
    for (int i = 0; i < n; ++i) {
        Pipeline& p = clouds[i]->p;
        if (p.prm.grid_lists && p.glist.valid && !p.glist.too_big) {
            listed[i] = 1;
            continue;
        }
        p.grid_batched = true;
        items.emplace_back();
        GwnBatchItem& it = items.back();
        it.tree = &p.t2;
        for (int d = 0; d < 3; ++d) {
            it.res[d] = p.gres[d];
            it.origin[d] = p.gorg[d];
        }
        it.spacing = p.gh;
        it.out = p.field.ptr;
        it.terms_total = p.terms_cur.ptr;
        it.sigma_dev = p.cur_sigma.ptr;
        it.beta = p.prm.beta;
    }
    unlisted = (int)items.size();
    if (unlisted) DWG_TRY(gwn_batch_prepare(grid, items.data(), unlisted, clouds[0]->p.gwn_params(), s));
    return DWG_OK;
}

// one iteration of every cloud on the batch stream, as one capture
int Batch::capture() {
    const int n = (int)clouds.size();
    DWG_CHECK_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    int st = DWG_OK;
    auto fail = [&](int code) {
        if (st == DWG_OK) st = code;
    };
    if (cudaEventRecord(ev_fork, s) != cudaSuccess) fail(DWG_ERR_CUDA);
    for (int i = 0; i < n && st == DWG_OK; ++i) {
        Pipeline& p = clouds[i]->p;
        if (cudaStreamWaitEvent(p.s, ev_fork, 0) != cudaSuccess) fail(DWG_ERR_CUDA);
        if (st == DWG_OK) fail(p.iterate_pre());
        if (listed[i]) {  // the whole iteration in this cloud's branch
            if (st == DWG_OK) fail(p.iterate_grid());
            if (st == DWG_OK) fail(p.iterate_post());
        }
        if (st == DWG_OK && cudaEventRecord(ev_done[i], p.s) != cudaSuccess) fail(DWG_ERR_CUDA);
        if (st == DWG_OK && cudaStreamWaitEvent(s, ev_done[i], 0) != cudaSuccess) fail(DWG_ERR_CUDA);
    }
    if (st == DWG_OK && unlisted) fail(gwn_batch_launch(grid, s));
    if (st == DWG_OK && cudaEventRecord(ev_mid, s) != cudaSuccess) fail(DWG_ERR_CUDA);
    for (int i = 0; i < n && st == DWG_OK; ++i) {
        Pipeline& p = clouds[i]->p;
        if (listed[i]) continue;
        if (cudaStreamWaitEvent(p.s, ev_mid, 0) != cudaSuccess) fail(DWG_ERR_CUDA);
        if (st == DWG_OK) fail(p.iterate_post());
        if (st == DWG_OK && cudaEventRecord(ev_done[n + i], p.s) != cudaSuccess) fail(DWG_ERR_CUDA);
        if (st == DWG_OK && cudaStreamWaitEvent(s, ev_done[n + i], 0) != cudaSuccess) fail(DWG_ERR_CUDA);
    }
    cudaGraph_t gr = nullptr;
    cudaError_t e = cudaStreamEndCapture(s, &gr);
    if (st != DWG_OK || e != cudaSuccess) {
        if (gr) cudaGraphDestroy(gr);
        if (st == DWG_OK) set_error("batch: capture failed: %s", cudaGetErrorString(e));
        return st != DWG_OK ? st : DWG_ERR_CUDA;
    }
    graph = gr;
    DWG_CHECK_CUDA(cudaGraphInstantiate(&graph_exec, graph, 0));
    return DWG_OK;
}

int Batch::iterate(int n_iters) {
    DWG_REQUIRE(!finalized, "batch: already finalized");
    if (n_iters <= 0) return DWG_OK;
    // history tables sized for the run; a reallocation invalidates the graph
    for (auto& c : clouds) {
        Pipeline& p = c->p;
        const int cap0 = p.hist_cap;
        DWG_TRY(p.ensure_hist(p.iter + n_iters));
        if (p.hist_cap != cap0 && graph_exec) {
            cudaGraphExecDestroy(graph_exec);
            cudaGraphDestroy(graph);
            graph_exec = nullptr;
            graph = nullptr;
        }
    }
    DWG_TRY(join_in());
    for (int k = 0; k < n_iters; ++k) {
        if (iter == 0) {
            // the first iteration runs eagerly per cloud: it sizes the
            // workspaces (marching cubes, kNN, repair) that the graph reuses
            // and records each cloud's grid lists (16 bytes per entry) within
            // what is left above the reserve, without weights: those (256
            // bytes per entry and sigma) are handed out once every cloud's
            // lists are known (prepare_grid)
            for (auto& c : clouds) {
                Pipeline& p = c->p;
                const size_t fr = device_free_bytes();
                const size_t room = fr > reserve ? fr - reserve : 0;
                p.glist_budget = std::min(p.glist_budget, room > 0 ? room : (size_t)1);
                p.glist.wmax = 1;
                DWG_TRY(p.iterate(1));
            }
        } else {
            if (!graph_exec) {
                DWG_TRY(prepare_grid());
                DWG_TRY(capture());
            }
            DWG_CHECK_CUDA(cudaGraphLaunch(graph_exec, s));
            for (auto& c : clouds) ++c->p.iter;
        }
        ++iter;
    }
    return join_out();
}

int Batch::finalize() {
    DWG_REQUIRE(!finalized, "batch: already finalized");
    DWG_TRY(join_in());
    // the iteration grids' lists and weights are done with: their memory
    // goes to the final passes (the batch stream waited for every cloud)
    DWG_CHECK_CUDA(cudaStreamSynchronize(s));
    {
        FreeScope idle(nullptr, true);
        for (auto& c : clouds) gwn_list_release(c->p.glist);
    }
    for (auto& c : clouds) DWG_TRY(c->p.finalize());
    finalized = true;
    return join_out();
}

}  // namespace dwg
