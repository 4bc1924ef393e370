// batch.cu -- many clouds reconstructed under one CUDA graph per iteration,
// with the grid sums of all clouds in one persistent launch.
#include "batch.cuh"

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
        // the batch's persistent launch sums the grids of later iterations;
        // lists of the first iteration's grid would only hold memory
        clouds.back()->p.grid_batched = true;
    }
    // the grid sums of every cloud, one work list
    std::vector<GwnBatchItem> items((size_t)n);
    for (int i = 0; i < n; ++i) {
        Pipeline& p = clouds[i]->p;
        GwnBatchItem& it = items[i];
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
    DWG_TRY(gwn_batch_prepare(grid, items.data(), n, clouds[0]->p.gwn_params(), s));
    return join_out();
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
        if (st == DWG_OK && cudaEventRecord(ev_done[i], p.s) != cudaSuccess) fail(DWG_ERR_CUDA);
        if (st == DWG_OK && cudaStreamWaitEvent(s, ev_done[i], 0) != cudaSuccess) fail(DWG_ERR_CUDA);
    }
    if (st == DWG_OK) fail(gwn_batch_launch(grid, s));
    if (st == DWG_OK && cudaEventRecord(ev_mid, s) != cudaSuccess) fail(DWG_ERR_CUDA);
    for (int i = 0; i < n && st == DWG_OK; ++i) {
        Pipeline& p = clouds[i]->p;
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
            for (auto& c : clouds) DWG_TRY(c->p.iterate(1));
        } else {
            if (!graph_exec) DWG_TRY(capture());
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
    for (auto& c : clouds) DWG_TRY(c->p.finalize());
    finalized = true;
    return join_out();
}

}  // namespace dwg
