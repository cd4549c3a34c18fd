// History output of the plain form: the writer the reference declares but
// never implements (runtime_params.c:24-27 reads SWE_OUTPUT_FILE and
// SWE_HIST_INT into sim_params; swe_config.h:112-115 names the field
// history_interval; nothing writes).
//
// Every `interval` completed RK4 steps the state is permuted into the
// caller's layout on the compute stream (the same data swe_cuda_get_state
// returns), copied to pinned host memory on a separate copy stream, and
// appended to the file by a writer thread, so the time loop never waits for
// the disk; it only waits when all kSlots snapshots are still in flight.
//
// File format (little endian):
//   header, 64 bytes: char magic[8] = "SWEHIST1"; int32 value_bytes (4 or 8);
//     int32 interval; int64 values per record; double dt; int32 layout flags
//     (bit 0 CFDL, bit 1 SFDL); int32 SIMD length; 24 bytes zero.
//   record: int64 step; double time (= step * dt); then the values.
#pragma once

#include <cuda_runtime.h>

#include <condition_variable>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <deque>
#include <mutex>
#include <string>
#include <thread>

#include "common.cuh"

namespace swe {

class HistoryWriter {
  public:
    static constexpr int kSlots = 4;

    HistoryWriter() = default;
    HistoryWriter(const HistoryWriter&) = delete;
    HistoryWriter& operator=(const HistoryWriter&) = delete;
    ~HistoryWriter() { close(); }   // a caller that never closed still gets its queued records

    bool active() const { return fp_ != nullptr; }
    int interval() const { return interval_; }
    long long records() {
        std::lock_guard<std::mutex> lk(mu_);
        return records_;
    }
    long long bytes() {
        std::lock_guard<std::mutex> lk(mu_);
        return bytes_;
    }

    int open(const char* path, int interval, long long nvalues, int value_bytes, double dt, int layout, int simd,
             int device) {
        if (active()) SWE_TRY(close());
        if (!path || interval <= 0) {
            set_error("swe_hist_open: need a path and interval >= 1");
            return SWE_ERR_ARG;
        }
        fp_ = std::fopen(path, "wb");
        if (!fp_) {
            set_error("swe_hist_open: cannot open %s for writing", path);
            return SWE_ERR_ARG;
        }
        interval_ = interval;
        nvalues_ = nvalues;
        rec_bytes_ = (size_t)nvalues * value_bytes;
        dt_ = dt;
        device_ = device;
        records_ = bytes_ = 0;
        failed_ = false;
        unsigned char hdr[64] = {};
        std::memcpy(hdr, "SWEHIST1", 8);
        const int32_t vb = value_bytes, iv = interval, lf = layout, sl = simd;
        const int64_t nv = nvalues;
        std::memcpy(hdr + 8, &vb, 4);
        std::memcpy(hdr + 12, &iv, 4);
        std::memcpy(hdr + 16, &nv, 8);
        std::memcpy(hdr + 24, &dt, 8);
        std::memcpy(hdr + 32, &lf, 4);
        std::memcpy(hdr + 36, &sl, 4);
        if (std::fwrite(hdr, 1, 64, fp_) != 64) {
            set_error("swe_hist_open: writing the header of %s failed", path);
            std::fclose(fp_);
            fp_ = nullptr;
            return SWE_ERR_ARG;
        }
        bytes_ = 64;
        SWE_CUDA_TRY(cudaStreamCreateWithFlags(&copy_, cudaStreamNonBlocking));
        for (Slot& s : slots_) {
            SWE_CUDA_TRY(cudaMalloc(&s.dbuf, rec_bytes_));
            SWE_CUDA_TRY(cudaMallocHost(&s.hbuf, rec_bytes_));
            SWE_CUDA_TRY(cudaEventCreateWithFlags(&s.filled, cudaEventDisableTiming));
            SWE_CUDA_TRY(cudaEventCreateWithFlags(&s.copied, cudaEventDisableTiming));
            s.busy = false;
        }
        stop_ = false;
        writer_ = std::thread([this] { run(); });
        return SWE_OK;
    }

    // After `step` completed RK4 steps (enqueued on `compute`): snapshot if due.
    // fill(dbuf) enqueues the copy of the state, in the caller's layout, into dbuf.
    template <typename Fill>
    int after_step(long long step, cudaStream_t compute, Fill fill) {
        if (!active() || step % interval_ != 0) return SWE_OK;
        int si = -1;
        {
            std::unique_lock<std::mutex> lk(mu_);
            cv_.wait(lk, [&] {
                for (int i = 0; i < kSlots; ++i)
                    if (!slots_[i].busy) return true;
                return failed_;
            });
            if (failed_) {
                set_error("history writer: %s", err_.c_str());
                return SWE_ERR_CUDA;
            }
            for (int i = 0; i < kSlots; ++i)
                if (!slots_[i].busy) { si = i; break; }
            slots_[si].busy = true;
        }
        Slot& s = slots_[si];
        // a failure after the slot was taken gives the slot back and marks the writer
        // failed, so that later snapshots report the error instead of waiting for a
        // slot that would never be freed
        int st = fill(s.dbuf);
        cudaError_t ce = cudaSuccess;
        const char* what = "filling a snapshot failed";
        if (st == SWE_OK) {
            if ((ce = cudaEventRecord(s.filled, compute)) != cudaSuccess ||
                (ce = cudaStreamWaitEvent(copy_, s.filled, 0)) != cudaSuccess ||
                (ce = cudaMemcpyAsync(s.hbuf, s.dbuf, rec_bytes_, cudaMemcpyDeviceToHost, copy_)) != cudaSuccess ||
                (ce = cudaEventRecord(s.copied, copy_)) != cudaSuccess) {
                st = SWE_ERR_CUDA;
                what = cudaGetErrorString(ce);
            }
        }
        if (st != SWE_OK) {
            {
                std::lock_guard<std::mutex> lk(mu_);
                s.busy = false;
                if (!failed_) {
                    failed_ = true;
                    err_ = what;
                }
            }
            cv_.notify_all();
            if (ce != cudaSuccess) set_error("history writer: %s", what);
            return st;
        }
        {
            std::lock_guard<std::mutex> lk(mu_);
            queue_.push_back({si, step});
        }
        cv_.notify_all();
        return SWE_OK;
    }

    // Writes every queued snapshot, closes the file and frees the buffers.
    int close() {
        if (!active()) return SWE_OK;
        {
            std::lock_guard<std::mutex> lk(mu_);
            stop_ = true;
        }
        cv_.notify_all();
        if (writer_.joinable()) writer_.join();
        bool failed;
        std::string err;
        {
            std::lock_guard<std::mutex> lk(mu_);
            failed = failed_;
            err = err_;
        }
        const bool closed_ok = std::fclose(fp_) == 0;
        fp_ = nullptr;
        for (Slot& s : slots_) {
            if (s.dbuf) cudaFree(s.dbuf);
            if (s.hbuf) cudaFreeHost(s.hbuf);
            if (s.filled) cudaEventDestroy(s.filled);
            if (s.copied) cudaEventDestroy(s.copied);
            s = Slot{};
        }
        if (copy_) cudaStreamDestroy(copy_);
        copy_ = nullptr;
        if (failed) {
            set_error("history writer: %s", err.c_str());
            return SWE_ERR_CUDA;
        }
        if (!closed_ok) {
            set_error("history writer: closing the file failed");
            return SWE_ERR_ARG;
        }
        return SWE_OK;
    }

  private:
    struct Slot {
        void* dbuf = nullptr;
        void* hbuf = nullptr;
        cudaEvent_t filled = nullptr, copied = nullptr;
        bool busy = false;
    };
    struct Job {
        int slot;
        long long step;
    };

    void run() {
        cudaSetDevice(device_);
        for (;;) {
            Job j;
            {
                std::unique_lock<std::mutex> lk(mu_);
                cv_.wait(lk, [&] { return stop_ || !queue_.empty(); });
                if (queue_.empty()) return;          // stop requested and nothing left
                j = queue_.front();
                queue_.pop_front();
            }
            Slot& s = slots_[j.slot];
            bool ok = cudaEventSynchronize(s.copied) == cudaSuccess;
            std::string why = ok ? "" : "a snapshot copy failed";
            bool failed_before;
            {
                std::lock_guard<std::mutex> lk(mu_);
                failed_before = failed_;
            }
            if (ok && !failed_before) {
                const int64_t step = j.step;
                const double t = (double)j.step * dt_;
                ok = std::fwrite(&step, 8, 1, fp_) == 1 && std::fwrite(&t, 8, 1, fp_) == 1 &&
                     std::fwrite(s.hbuf, 1, rec_bytes_, fp_) == rec_bytes_;
                if (!ok) why = "writing a record failed";
            }
            {
                std::lock_guard<std::mutex> lk(mu_);
                if (ok) {
                    ++records_;
                    bytes_ += 16 + (long long)rec_bytes_;
                } else if (!failed_) {
                    failed_ = true;
                    err_ = why;
                }
                s.busy = false;
            }
            cv_.notify_all();
        }
    }

    FILE* fp_ = nullptr;
    int interval_ = 0, device_ = 0;
    long long nvalues_ = 0, records_ = 0, bytes_ = 0;
    size_t rec_bytes_ = 0;
    double dt_ = 0.0;
    cudaStream_t copy_ = nullptr;
    Slot slots_[kSlots];
    std::thread writer_;
    std::mutex mu_;
    std::condition_variable cv_;
    std::deque<Job> queue_;
    bool stop_ = false, failed_ = false;
    std::string err_;
};

}  // namespace swe
