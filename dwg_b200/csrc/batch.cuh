// batch.cuh -- many clouds of uneven size reconstructed together.
//
// Every cloud is a Pipeline with its own stream.  In the first iteration
// (eager, cloud by cloud) each cloud records its grid's interaction lists and
// keeps screening weights while they fit a memory budget shared by the
// batch.  Every later iteration of all clouds is one CUDA graph: a cloud with
// kept lists runs its whole iteration as its own branch; the grids of the
// others are summed by one persistent launch (a shared work list of bricks,
// so small clouds do not leave SMs idle) between their branches' phases.
#pragma once

#include <memory>
#include <vector>

#include "pipeline.cuh"

struct dwg_pipeline {
    dwg::Pipeline p;
};

namespace dwg {

struct Batch {
    std::vector<std::unique_ptr<dwg_pipeline>> clouds;
    cudaStream_t s = nullptr;       // the batch's stream (graph launches)
    cudaStream_t caller = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_mid = nullptr;
    std::vector<cudaEvent_t> ev_done;
    GwnBatch grid;
    std::vector<char> listed;       // per cloud: its grid replays kept lists in its own branch
    int unlisted = 0;               // clouds summed by the persistent launch
    size_t reserve = 0;             // bytes kept free for the first iteration's workspaces
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t graph_exec = nullptr;
    int iter = 0;
    bool finalized = false;

    ~Batch();
    // params[i]: the flags of cloud i (in_normal 3; tile must agree)
    int setup(const float* const* points_dev, const int* counts, int n, const dwg_params* params,
              cudaStream_t stream);
    int iterate(int n_iters);
    int finalize();

  private:
    int capture();
    int prepare_grid();
    int join_in();
    int join_out();
};

}  // namespace dwg
