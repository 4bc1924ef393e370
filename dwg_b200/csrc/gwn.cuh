// gwn.cuh -- generalised winding number sums over the octree.
#pragma once

#include "octree.cuh"

namespace dwg {

struct GwnQuery {
    // point queries (packed xyz) ...
    const float* q = nullptr;
    long long nq = 0;
    // ... or a regular grid (q == nullptr)
    int res[3] = {0, 0, 0};
    float origin[3] = {0, 0, 0};
    float spacing = 0;
    int zoff = 0;  // grid: z index of the first sample (a slab of a larger grid)
};

// out[i] = w(q_i); terms_total (nullable) += number of evaluated terms;
// per_query_terms (nullable) receives the count per query.
// sigma_dev (nullable) overrides p.sigma with a device value (graph replay).
int gwn_eval(const Octree& t, const GwnQuery& q, const dwg_gwn_params& p, float* out,
             unsigned long long* terms_total, int* per_query_terms, cudaStream_t s,
             const float* sigma_dev = nullptr);

// Interaction lists of a grid sum.  The Barnes-Hut decisions of a grid
// sample depend only on the tree's positions, areas and opening thresholds
// and on the sample, not on the normals or sigma, so in the DWG loop (fixed
// leaves, fixed grid) every iteration repeats the same traversal.  The first
// call records, per group of samples, the visits where some sample takes a
// term -- (record, per-slot lane masks), 16 bytes each -- and every later
// call replays them: the same terms in the same order, bit-identical sums,
// without the traversal.  A list larger than max_bytes is not kept (the sums
// then traverse every time).  The first call synchronises the stream.
//
// Screening weights: a far-node term is g (A n).(p - q) with
// g = |sigma rho + 1| / (e^{sigma rho} 4 pi rho^3 + 1e-7), which depends on
// the geometry and sigma only.  With weight slots, the replay also keeps g
// per node entry and sample (8 bytes per entry and lane) for up to
// kGwnWeightSlots values of (sigma, screen): a launch whose sigma has a slot
// reads g and skips the screening arithmetic (same bits); one without writes
// the next free slot while it evaluates.  The choice is made on the device
// (GwnWeightState), so CUDA graph replays with a device sigma work.
constexpr int kGwnWeightSlots = 4;
struct GwnWeightState {
    int mode, slot, nslots, pad;  // mode: 0 evaluate, 1 evaluate and write slot, 2 read slot
    int valid[kGwnWeightSlots];
    float sigma[kGwnWeightSlots], screen[kGwnWeightSlots];
    float pref[kGwnWeightSlots];  // the sigma a free slot is kept for (0: any)
    unsigned long long node_terms[kGwnWeightSlots];  // node terms a slot stands for
    unsigned int work;                               // group counter of the reading launch
};

struct GwnList {
    DevBuf<unsigned int> count;          // entries per group (recording)
    DevBuf<unsigned long long> off;      // first entry of each group, ngroups + 1
    DevBuf<int4> ent;                    // the entries
    DevBuf<unsigned char> scratch;
    DevBuf<float2> w;                    // weight slots, nslots * entries * 32
    DevBuf<GwnWeightState> wstate;
    int wslots = 0;                      // weight slots wanted (0: none)
    int nslots = 0;                      // weight slots held
    size_t wmax = 0;                     // entries and weights together at most this many bytes (0: no such cap)
    // when fewer slots are held than wanted, slot c is kept for sigma pref[c]
    // (the owner's most used sigmas first; 0: the first sigma that comes)
    float pref[kGwnWeightSlots] = {0.f, 0.f, 0.f, 0.f};
    long long ngroups = 0;
    unsigned long long entries = 0;
    // what the recorded decisions depend on besides the tree's centres (the
    // positions of point queries are the caller's to keep: same pointer, same
    // points)
    bool grid = true;
    const float* qptr = nullptr;
    long long nq = 0;
    int tile = -1, res[3] = {0, 0, 0}, zoff = 0, use_radii = 0;
    float origin[3] = {0, 0, 0}, spacing = 0, beta = 0;
    bool valid = false, too_big = false;
    GwnList() = default;
    GwnList(const GwnList&) = delete;
    GwnList& operator=(const GwnList&) = delete;
    ~GwnList();
};

// screened sums at a grid or at points through L (recorded on the first
// call, recorded again when the grid, the query pointer or count, tile, beta
// or use_radii differ); the caller resets L.valid when the tree's centres of
// mass or the query points change.  A list above max_bytes (0: a
// quarter of the free memory when it is recorded) is not kept.  wslots > 0
// keeps screening weights for up to that many (sigma, screen) values (at most
// kGwnWeightSlots; slots that do not fit in a third of the free memory, or
// 64 GB, are dropped) when the terms use the MUFU approximations (precision
// 0 or 1).
int gwn_eval_listed(const Octree& t, const GwnQuery& q, const dwg_gwn_params& p, GwnList& L, float* out,
                    unsigned long long* terms_total, cudaStream_t s, const float* sigma_dev, size_t max_bytes,
                    int wslots = 0);

// Values and/or gradients (out_g: 3 per query) of the sums, one thread per
// query with the decisions of gwn_eval; fp64: terms and sums in double from
// the FP64 moments (outputs double), else FP32 terms summed in double
// (outputs float).  Order-0 far field only.
int gwn_eval_thread(const Octree& t, const GwnQuery& q, const dwg_gwn_params& p, bool fp64, void* out_w,
                    void* out_g, cudaStream_t s);

// Frees every weight slot of L (the list itself stays): the kept weights
// depend on the points' screening radii when use_radii is set, so new radii
// make them stale.  Stream-ordered, no host synchronisation.
int gwn_list_drop_weights(GwnList& L, cudaStream_t s);
// weight slots for a kept list that holds none yet (nslots <= L.wslots),
// written by the next replay of each sigma; DWG_ERR_NOMEM leaves it without
int gwn_list_add_weights(GwnList& L, int nslots, cudaStream_t s);
// give back a list's memory (entries and weights); the next call records again
void gwn_list_release(GwnList& L);

// Grid sums of many clouds in one persistent launch (screened).  prepare()
// records the clouds' octrees, grids and outputs once (host work, not
// capturable); launch() is two stream operations and can be captured in a
// CUDA graph and replayed while the octrees' moments change in place.
struct GwnBatchItem {
    Octree* tree = nullptr;
    int res[3] = {0, 0, 0};
    float origin[3] = {0, 0, 0};
    float spacing = 0;
    float* out = nullptr;
    unsigned long long* terms_total = nullptr;  // nullable
    const float* sigma_dev = nullptr;           // nullable: p.sigma
    float beta = 0.f;                           // opening ratio of this cloud (0: p.beta)
};

struct GwnBatchImpl;
struct GwnBatch {
    GwnBatchImpl* impl = nullptr;
    unsigned long long groups = 0;
    GwnBatch() = default;
    GwnBatch(const GwnBatch&) = delete;
    GwnBatch& operator=(const GwnBatch&) = delete;
    ~GwnBatch();
};

int gwn_batch_prepare(GwnBatch& b, const GwnBatchItem* items, int n, const dwg_gwn_params& p, cudaStream_t s);
int gwn_batch_launch(GwnBatch& b, cudaStream_t s);

}  // namespace dwg
