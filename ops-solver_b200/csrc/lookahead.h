// lookahead.h -- look-ahead for the blocked QR factorisations: the panel chain (panel, T,
// the update of the next panel's columns) runs on a stream of the device's greatest priority
// forked from the caller's stream, while the wide trailing update stays on the caller's
// stream, so each panel overlaps the previous panel's wide update.  Events order the two.
#pragma once
#include <cuda_runtime.h>

namespace ops_solver
{
class Lookahead
{
  public:
    cudaStream_t panel = nullptr;

    Lookahead() = default;
    Lookahead(const Lookahead &) = delete;
    Lookahead &operator=(const Lookahead &) = delete;
    ~Lookahead() { release(); }

    // Creates the panel stream and forks it from s.
    cudaError_t open(cudaStream_t s)
    {
        int least = 0, greatest = 0;
        cudaError_t e = cudaDeviceGetStreamPriorityRange(&least, &greatest);
        if (e == cudaSuccess) e = cudaStreamCreateWithPriority(&panel, cudaStreamNonBlocking, greatest);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&to_main_, cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&to_panel_, cudaEventDisableTiming);
        if (e == cudaSuccess) e = to_panel(s);
        return e;
    }
    // s waits for the panel stream's work so far.
    cudaError_t to_main(cudaStream_t s)
    {
        cudaError_t e = cudaEventRecord(to_main_, panel);
        return e == cudaSuccess ? cudaStreamWaitEvent(s, to_main_, 0) : e;
    }
    // The panel stream waits for s's work so far.
    cudaError_t to_panel(cudaStream_t s)
    {
        cudaError_t e = cudaEventRecord(to_panel_, s);
        return e == cudaSuccess ? cudaStreamWaitEvent(panel, to_panel_, 0) : e;
    }
    // Joins the panel stream back into s and releases both streams' helpers (the device
    // finishes the queued work first).
    cudaError_t close(cudaStream_t s)
    {
        cudaError_t e = to_main(s);
        release();
        return e;
    }
    // Gives up after a failed open (nothing but the fork is queued on the panel stream); the
    // caller then runs without look-ahead.
    void abandon()
    {
        cudaGetLastError();
        release();
    }

  private:
    cudaEvent_t to_main_ = nullptr, to_panel_ = nullptr;

    void release()
    {
        if (to_main_) cudaEventDestroy(to_main_);
        if (to_panel_) cudaEventDestroy(to_panel_);
        if (panel) cudaStreamDestroy(panel);
        to_main_ = to_panel_ = nullptr;
        panel = nullptr;
    }
};
}  // namespace ops_solver
