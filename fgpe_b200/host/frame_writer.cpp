// frame_writer.cpp -- asynchronous psi.wdat frame appends for the host mirror.
//
// The reference appends a frame every itmod iterations by a blocking device
// copy followed by a file write (hamiltonians/BEC_oneComponent.cu:361-365,
// src/output.cu:193-197), so the GPU idles while the disk is written.  Here
// each frame is converted to complex128 on the device (gpe_get_psi_device),
// copied into one of two pinned host slots on the solver's stream, and
// appended to the same file by a writer thread once the copy's event has
// completed; the stepping loop continues meanwhile.  The bytes and their
// order in the file are those of the synchronous path.
#include <cuda_runtime.h>

#include "gpe_host.hpp"

namespace gpe {

namespace {
void cuda_chk(cudaError_t e, const char* what) {
    if (e != cudaSuccess) throw HostError(std::string(what) + ": " + cudaGetErrorString(e));
}
}  // namespace

FrameWriter::~FrameWriter() {
    try {
        flush();
    } catch (...) {
        // a write error is reported by flush() to the solver's run loop; a
        // destructor must not throw
    }
    {
        std::lock_guard<std::mutex> lk(m_);
        stop_ = true;
    }
    cv_.notify_all();
    if (thread_.joinable()) thread_.join();
    for (int s = 0; s < 2; ++s) {
        if (host_[s]) cudaFreeHost(host_[s]);
        if (ev_[s]) cudaEventDestroy((cudaEvent_t)ev_[s]);
    }
    if (dev_) cudaFree(dev_);
}

void FrameWriter::start(Output* out, gpe_handle* h, long long n, int ncomp) {
    out_ = out;
    h_ = h;
    n_ = n;
    ncomp_ = ncomp;
    const size_t bytes = sizeof(complex) * (size_t)n * (size_t)ncomp;
    cuda_chk(cudaMalloc(&dev_, bytes), "frame writer: cudaMalloc");
    for (int s = 0; s < 2; ++s) {
        cuda_chk(cudaMallocHost(&host_[s], bytes), "frame writer: cudaMallocHost");
        cudaEvent_t e = nullptr;
        cuda_chk(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "frame writer: cudaEventCreate");
        ev_[s] = e;
    }
    thread_ = std::thread([this] { run(); });
}

void FrameWriter::push(const std::vector<std::string>& suffixes) {
    if ((int)suffixes.size() != ncomp_) throw HostError("frame writer: one file suffix per component");
    std::unique_lock<std::mutex> lk(m_);
    if (err_) std::rethrow_exception(err_);
    cv_.wait(lk, [&] { return !busy_[slot_] || err_; });
    if (err_) std::rethrow_exception(err_);
    const int s = slot_;
    lk.unlock();
    // The solver's handle runs on the default stream: the conversion, the
    // copy and the event are ordered after the steps that produced the frame,
    // and the next frame's conversion after this copy has read dev_.
    for (int c = 0; c < ncomp_; ++c) {
        complex* d = (complex*)dev_ + c * (size_t)n_;
        const gpe_status st = gpe_get_psi_device(h_, c, d);
        if (st != GPE_OK) throw HostError(std::string("gpe_get_psi_device: ") + gpe_last_error_string());
        cuda_chk(cudaMemcpyAsync((complex*)host_[s] + c * (size_t)n_, d, sizeof(complex) * (size_t)n_,
                                 cudaMemcpyDeviceToHost, 0),
                 "frame writer: cudaMemcpyAsync");
    }
    cuda_chk(cudaEventRecord((cudaEvent_t)ev_[s], 0), "frame writer: cudaEventRecord");
    lk.lock();
    busy_[s] = true;
    queue_.push_back(Frame{s, suffixes});
    slot_ = 1 - s;
    lk.unlock();
    cv_.notify_all();
}

void FrameWriter::flush() {
    std::unique_lock<std::mutex> lk(m_);
    cv_.wait(lk, [&] { return queue_.empty(); });
    if (err_) {
        std::exception_ptr e = err_;
        err_ = nullptr;
        std::rethrow_exception(e);
    }
}

void FrameWriter::run() {
    std::unique_lock<std::mutex> lk(m_);
    for (;;) {
        cv_.wait(lk, [&] { return stop_ || !queue_.empty(); });
        if (queue_.empty()) return;  // stop_ with nothing left
        const Frame f = queue_.front();
        const int s = f.slot;
        lk.unlock();
        std::exception_ptr e;
        try {
            cuda_chk(cudaEventSynchronize((cudaEvent_t)ev_[s]), "frame writer: cudaEventSynchronize");
            for (int c = 0; c < ncomp_; ++c)
                out_->WritePsi((const complex*)host_[s] + c * (size_t)n_, (int)n_, f.suffixes[c]);
        } catch (...) {
            e = std::current_exception();
        }
        lk.lock();
        if (e && !err_) err_ = e;
        queue_.pop_front();
        busy_[s] = false;
        cv_.notify_all();
    }
}

}  // namespace gpe
