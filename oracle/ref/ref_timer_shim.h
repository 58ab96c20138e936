// Headless stand-in for the reference's core/utilities.h, used only when the
// reference kernels are compiled into oracle/_ref for parity checks.
//
// core/utilities.h:155-187 defines CudaTimer (an event pair whose stop()
// blocks on cudaEventSynchronize) next to OpenGL buffer wrappers.  The
// kernels in core/gaussian_render.cu only use CudaTimer, so this header
// provides that class with the same members and the same blocking
// semantics, and nothing else.  No graphics header is involved.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include <glm/glm.hpp>
#include <vector>
#include "cuda_error_check.cpp"

struct CudaTimer
{
  private:
    cudaEvent_t m_Start;
    cudaEvent_t m_Stop;
    float m_ElapsedTimeMs{0};

  public:
    CudaTimer()
    {
        cudaEventCreate(&m_Start);
        cudaEventCreate(&m_Stop);
    }
    ~CudaTimer()
    {
        cudaEventDestroy(m_Start);
        cudaEventDestroy(m_Stop);
    }
    void start() { cudaEventRecord(m_Start); }
    void stop()
    {
        cudaEventRecord(m_Stop);
        cudaEventSynchronize(m_Stop);
        cudaEventElapsedTime(&m_ElapsedTimeMs, m_Start, m_Stop);
    }
    float getElapseTimedMs() const { return m_ElapsedTimeMs; }
};
