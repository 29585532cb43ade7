// Host-side I/O of the C ABI: parallel file reads into pinned staging and
// the host buffers of query results.  Plain C++ (POSIX), no CUDA, so the
// test suite exercises it on the CPU.
#pragma once

#include <fcntl.h>
#include <sys/types.h>
#include <unistd.h>

#include <algorithm>
#include <cerrno>
#include <condition_variable>
#include <cstdint>
#include <cstring>
#include <mutex>
#include <new>
#include <thread>
#include <vector>

namespace gpj {

// Reads byte ranges of a file into host memory with up to `threads`
// threads: each range is cut into one slice per thread, read concurrently
// by preads.  A file load is bound by this copy out of the page cache,
// which one thread does at a fraction of host memory bandwidth.  The
// workers live for one load, so a range costs two condition-variable
// round trips, not thread starts.
class SliceReader {
  public:
    SliceReader(int fd, int threads) : fd_(fd) {
        try {
            for (int i = 1; i < threads; i++) workers_.emplace_back([this, i] { work(i); });
        } catch (const std::exception&) {
            // fewer threads than asked: the ranges are cut into fewer slices
        }
        parts_ = static_cast<int>(workers_.size()) + 1;
    }

    ~SliceReader() {
        {
            std::lock_guard<std::mutex> g(mu_);
            quit_ = true;
        }
        go_.notify_all();
        for (auto& t : workers_) t.join();
    }

    // Bytes [pos, pos + len) into dst; false on an I/O error or a short
    // read (the file shrank).
    bool read(uint8_t* dst, int64_t pos, size_t len) {
        {
            std::lock_guard<std::mutex> g(mu_);
            dst_ = dst;
            pos_ = pos;
            len_ = len;
            ok_ = true;
            pending_ = parts_ - 1;
            ++round_;
        }
        go_.notify_all();
        const bool mine = read_slice(0);
        std::unique_lock<std::mutex> g(mu_);
        done_.wait(g, [this] { return pending_ == 0; });
        return mine && ok_;
    }

  private:
    // Slice i of the current range (the range is fixed until every slice is read).
    bool read_slice(int i) const {
        const size_t slice = (len_ + parts_ - 1) / parts_;
        const size_t off = std::min(len_, slice * static_cast<size_t>(i));
        const size_t want = std::min(slice, len_ - off);
        size_t got = 0;
        while (got < want) {
            const ssize_t r = ::pread(fd_, dst_ + off + got, want - got, static_cast<off_t>(pos_ + off + got));
            if (r < 0 && errno == EINTR) continue;
            if (r <= 0) return false;
            got += static_cast<size_t>(r);
        }
        return true;
    }

    void work(int i) {
        uint64_t seen = 0;
        for (;;) {
            {
                std::unique_lock<std::mutex> g(mu_);
                go_.wait(g, [&] { return quit_ || round_ != seen; });
                if (quit_) return;
                seen = round_;
            }
            const bool ok = read_slice(i);
            {
                std::lock_guard<std::mutex> g(mu_);
                ok_ = ok_ && ok;
                --pending_;
            }
            done_.notify_one();
        }
    }

    const int fd_;
    int parts_ = 1;
    std::vector<std::thread> workers_;
    std::mutex mu_;
    std::condition_variable go_, done_;
    uint64_t round_ = 0;
    int pending_ = 0;
    bool ok_ = true, quit_ = false;
    uint8_t* dst_ = nullptr;
    int64_t pos_ = 0;
    size_t len_ = 0;
};

// Host memory for results.  A new buffer's first touch (page faults) costs
// several times the device-to-host copy into it, and a copy that faults in
// its own pages is slower still, so the largest released buffer (up to
// kKeepElems) is kept for the next result of the process, and a new one is
// touched once before the copy.
class ResultBuffers {
  public:
    static constexpr size_t kKeepElems = size_t(64) << 20;  // 512 MiB

    int64_t* take(size_t count, size_t* cap) {
        {
            std::lock_guard<std::mutex> g(mu_);
            if (kept_ && kept_cap_ >= count) {
                int64_t* p = kept_;
                *cap = kept_cap_;
                kept_ = nullptr;
                kept_cap_ = 0;
                return p;
            }
        }
        int64_t* p = new (std::nothrow) int64_t[count];
        if (p) std::memset(p, 0, count * sizeof(int64_t));
        *cap = count;
        return p;
    }

    void give(int64_t* p, size_t cap) {
        if (!p) return;
        {
            std::lock_guard<std::mutex> g(mu_);
            if (cap <= kKeepElems && cap > kept_cap_) {
                std::swap(p, kept_);
                std::swap(cap, kept_cap_);
            }
        }
        delete[] p;
    }

    ResultBuffers() = default;
    ResultBuffers(const ResultBuffers&) = delete;
    ResultBuffers& operator=(const ResultBuffers&) = delete;
    ~ResultBuffers() { delete[] kept_; }

  private:
    std::mutex mu_;
    int64_t* kept_ = nullptr;
    size_t kept_cap_ = 0;
};

// Never destroyed, so that results released during process exit find it.
inline ResultBuffers& result_buffers() {
    static ResultBuffers* b = new ResultBuffers;
    return *b;
}

}  // namespace gpj
