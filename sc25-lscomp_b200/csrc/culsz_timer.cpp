// culsz_timer.cpp -- TimingGPU (include/cuLSZ_timer.h): CUDA-event timing on
// the legacy default stream, the scope the reference's CLIs time
// (lsCOMP/src/cuLSZ_timer.cu).  The two events are created once per timer
// and destroyed with it.
#include "cuLSZ_timer.h"

TimingGPU::TimingGPU()
{
    privateTimingGPU = new PrivateTimingGPU;
    cudaEventCreate(&privateTimingGPU->start);
    cudaEventCreate(&privateTimingGPU->stop);
}

TimingGPU::~TimingGPU()
{
    cudaEventDestroy(privateTimingGPU->start);
    cudaEventDestroy(privateTimingGPU->stop);
    delete privateTimingGPU;
}

void TimingGPU::StartCounter() { cudaEventRecord(privateTimingGPU->start, 0); }

// Same as StartCounter but with blocking-sync events (the waiting host thread
// sleeps instead of spinning).
void TimingGPU::StartCounterFlags()
{
    cudaEventDestroy(privateTimingGPU->start);
    cudaEventDestroy(privateTimingGPU->stop);
    cudaEventCreateWithFlags(&privateTimingGPU->start, cudaEventBlockingSync);
    cudaEventCreateWithFlags(&privateTimingGPU->stop, cudaEventBlockingSync);
    cudaEventRecord(privateTimingGPU->start, 0);
}

float TimingGPU::GetCounter()
{
    float ms = 0.f;
    cudaEventRecord(privateTimingGPU->stop, 0);
    cudaEventSynchronize(privateTimingGPU->stop);
    cudaEventElapsedTime(&ms, privateTimingGPU->start, privateTimingGPU->stop);
    return ms;
}
