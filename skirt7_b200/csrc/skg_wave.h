// skg_wave.h -- host side of the wavefront packet tracer (kernels in skg_tracer.cu).
//
// A phase runs as a sequence of waves on one stream.  Wave w: an event pass over the packet pool
// (detect the previous wave's peel-offs, launch new packets into free records, move scattered
// packets to their interaction point, scatter, and write the next traversals as jobs) followed by
// a traversal pass that walks every job of the wave.  The number of waves is not known in
// advance: begin() enqueues an estimate, finish() reads how many packets still had work after the
// last enqueued wave and enqueues more until none has -- or, once few have, the tail pass, which
// finishes every remaining packet in one launch.
#pragma once
#include "skg_scene.cuh"

#include <vector>

namespace skg {

class WaveRunner {
public:
    WaveRunner() = default;
    WaveRunner(const WaveRunner&) = delete;
    WaveRunner& operator=(const WaveRunner&) = delete;
    ~WaveRunner();

    // Sizes the pool and job buffers (allocates; call outside stream capture).  pool packets,
    // ngroups peel-off groups at most per packet; grid_type decides whether path walks keep
    // checkpoints (grids whose FP32 walk resumes).
    cudaError_t reserve(size_t pool, int ngroups, int grid_type);
    // Enqueues the reset of the pool and the first waves of a phase on stream s.  P holds the
    // staged tables; nslots the slots whose DevGrid the traversal pass keeps in shared memory;
    // tree_walk the FP32 tree walk (TreeWalk) of tree grids; one_grid (host copy), when given with
    // nslots = 1, the grid the FP32 traversal kernels take as a kernel parameter instead.
    cudaError_t begin(const RunParams& P, int grid_type, int tree_walk, int precision, int nslots,
                      size_t npool, int trav_blocks, cudaStream_t s, const DevGrid* one_grid = nullptr);
    // Waits for the enqueued waves and enqueues more until no packet is left; then records
    // `end` (if given) on the phase's stream.  timeout_ms < 0 waits without limit.
    cudaError_t finish(int timeout_ms, cudaEvent_t end, bool* timed_out);
    // A captured begin() (pool reset and n waves) was launched as a graph on stream s.
    void replayed(cudaStream_t s, int n) { pending_ = true; stream_ = s; waves_ = n; }
    bool pending() const { return pending_; }
    int waves() const { return waves_; }
    size_t pool_capacity() const { return cap_pool_; }
    // With timing on, each wave's two kernels are bracketed by events (not inside graph capture).
    bool timing = false;
    // Device time of the finished phase's event passes and traversal passes (ms).
    cudaError_t times(float* event_ms, float* trav_ms) const;

    int estimate = 24;                // waves the next phase enqueues up front
    // the tail pass takes over when at most npool / tail_div packets had work in the last wave
    // (0: waves to the end; the environment variable SKG_TAIL_DIV overrides it per phase)
    int tail_div = 16;

private:
    cudaError_t enqueue(int n);
    cudaError_t enqueue_tail();

    Packet* pk_ = nullptr;
    int* free_ = nullptr;             // [pool] records freed in a wave, [pool] records at their
                                      // interaction point (the scatter-and-launch pass's work)
    float4* ckpt_ = nullptr;          // [pool][checkpoints][2] path-walk checkpoints
    size_t cap_ckpt_ = 0;
    size_t cap_pool_ = 0;
    int2* jobs_[2] = {nullptr, nullptr};
    double* jtau_[2] = {nullptr, nullptr};
    double* jL_[2] = {nullptr, nullptr};
    size_t cap_jobs_ = 0;
    static constexpr int NCTR = 17;
    unsigned* ctr_ = nullptr;         // [8b .. 8b+7]: counters of job buffer b; [16]: last busy wave
    unsigned* h_ctr_ = nullptr;       // pinned copy read by finish()
    cudaEvent_t copied_ = nullptr;

    bool pending_ = false;
    cudaStream_t stream_ = nullptr;
    RunParams P_{};
    int grid_type_ = 0, precision_ = 0, nslots_ = 1, trav_blocks_ = 0;
    bool one_ = false;                 // a single-slot launch with its grid in g0_
    DevGrid g0_{};
    int tree_walk_ = TW_ROPE;
    int npool_ = 0;
    int waves_ = 0;
    std::vector<cudaEvent_t> ev_;      // 3 per wave: before the event pass, between, after the traversal
    bool timed_ = false;               // the running phase records ev_
    int tail_div_ = 16;
    bool ckpt_on_ = true;              // path-walk checkpoints (environment variable SKG_CKPT=0: off)
    bool tail_ran_ = false;            // the phase ended with the tail pass
    cudaEvent_t tail_ev_[2] = {nullptr, nullptr};
};

}  // namespace skg
