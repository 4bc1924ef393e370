// batch.cuh -- many clouds of uneven size reconstructed together.
//
// Every cloud is a Pipeline with its own stream.  One iteration of all
// clouds is captured once as a single CUDA graph: the per-cloud phases
// before the grid sums run as parallel branches, the grid sums of all clouds
// are one persistent launch (a shared work list of bricks, so small clouds do
// not leave SMs idle), and the per-cloud phases after it branch out again.
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
    int join_in();
    int join_out();
};

}  // namespace dwg
