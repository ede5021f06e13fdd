// TimeAcc of mcstar-libs cuda/cutiming.hpp:5-25: accumulates the device time between
// start() and stop() (CUDA events on the legacy default stream) over repeated
// intervals; streaming it prints the total in milliseconds.
#pragma once
#include <cuda_runtime.h>

#include <ostream>

class TimeAcc {
    cudaEvent_t m_starte, m_ende;
    int m_times;
    float m_elapsed_ms;

  public:
    TimeAcc() : m_times(1), m_elapsed_ms(0.f) {
        cudaEventCreate(&m_starte);
        cudaEventCreate(&m_ende);
    }
    ~TimeAcc() {
        cudaEventDestroy(m_starte);
        cudaEventDestroy(m_ende);
    }
    TimeAcc(const TimeAcc&) = delete;
    TimeAcc& operator=(const TimeAcc&) = delete;
    void start() { cudaEventRecord(m_starte); }
    void stop(bool incr = true) {
        cudaEventRecord(m_ende);
        cudaEventSynchronize(m_ende);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, m_starte, m_ende);
        if (incr) m_times++;
        m_elapsed_ms += ms;
    }
    void reset() {
        m_times = 1;
        m_elapsed_ms = 0.f;
    }
    friend std::ostream& operator<<(std::ostream& o, const TimeAcc& t) { return o << t.m_elapsed_ms; }
};
