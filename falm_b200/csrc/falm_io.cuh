// Output formats of the reference's time loop (src/FalmIO.h, src/falm.h:433-478):
// snapshot vector files, the index JSON, control-volume files, and the running
// time average.
//
// Snapshots leave the GPU without stopping the time loop: the columns are
// copied on the caller's stream into one of two pinned staging buffers (cast to
// FP64 on the device first when asked), an event marks the copy, and a host
// thread of the context waits for the event and writes the file.  A third
// snapshot waits for one of the two buffers to be free; falm_io_wait() waits for
// every queued file.
#pragma once
#include <condition_variable>
#include <cstdint>
#include <deque>
#include <string>
#include <thread>
#include <charconv>
#include "falm_internal.cuh"

namespace fb {

// one column block of an FP32 field cast to FP64 (the snapshot's as_fp64 option)
__global__ void k_cast_f64(const float *__restrict__ src, double *__restrict__ dst, long long n) {
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x)
        dst[q] = (double)src[q];
}

struct IoBuf {
    void *host = nullptr;      // pinned
    void *dev = nullptr;       // FP64 staging of the cast option
    size_t cap = 0, dcap = 0;
    bool in_use = false;
    cudaEvent_t ready = nullptr;
};

struct IoJob {
    std::string path;
    uint64_t head[6];          // imax, jmax, kmax, ncol, gc, step
    double time;
    uint64_t dsize;
    size_t bytes;
    int buf;
};

struct IoWriter {
    int device = 0;
    std::mutex m;
    std::condition_variable cv;
    std::deque<IoJob> jobs;
    std::thread worker;
    bool stop = false;
    int pending = 0;           // jobs queued or being written
    int error = 0;             // first error since the last falm_io_wait
    std::string error_msg;
    IoBuf bufs[2];

    void run() {
        cudaSetDevice(device);
        for (;;) {
            IoJob job;
            {
                std::unique_lock<std::mutex> lk(m);
                cv.wait(lk, [&] { return stop || !jobs.empty(); });
                if (jobs.empty()) return;
                job = jobs.front();
                jobs.pop_front();
            }
            IoBuf &b = bufs[job.buf];
            int rc = 0;
            std::string msg;
            if (cudaEventSynchronize(b.ready) != cudaSuccess) {
                rc = FALM_ERR_CUDA;
                msg = "snapshot copy failed";
            } else {
                FILE *f = fopen(job.path.c_str(), "wb");
                bool ok = f != nullptr;
                ok = ok && fwrite(job.head, sizeof(uint64_t), 6, f) == 6;
                ok = ok && fwrite(&job.time, sizeof(double), 1, f) == 1;
                ok = ok && fwrite(&job.dsize, sizeof(uint64_t), 1, f) == 1;
                ok = ok && fwrite(b.host, 1, job.bytes, f) == job.bytes;
                if (f && fclose(f) != 0) ok = false;
                if (!ok) { rc = FALM_ERR_ARG; msg = "cannot write " + job.path; }
            }
            {
                std::lock_guard<std::mutex> lk(m);
                b.in_use = false;
                pending--;
                if (rc && !error) { error = rc; error_msg = msg; }
            }
            cv.notify_all();
        }
    }

    ~IoWriter() {
        {
            std::lock_guard<std::mutex> lk(m);
            stop = true;
        }
        cv.notify_all();
        if (worker.joinable()) worker.join();
        for (IoBuf &b : bufs) {
            if (b.host) cudaFreeHost(b.host);
            if (b.dev) cudaFree(b.dev);
            if (b.ready) cudaEventDestroy(b.ready);
        }
    }
};

// nlohmann::json's rendering of a double (the reference writes its index file
// with it): the shortest round-trip digits d1..dk with decimal exponent n
// (value = 0.d1..dk x 10^n), written as
//   k <= n <= 15 : the digits, n - k zeros, ".0"
//   0 < n <= 15  : the digits with the point after n of them
//   -4 < n <= 0  : "0." then -n zeros, then the digits
//   otherwise    : d1[.d2..dk]e(+|-)XX, at least two exponent digits
inline std::string json_double(double v) {
    if (v == 0.0) return std::signbit(v) ? "-0.0" : "0.0";
    char buf[64];
    auto res = std::to_chars(buf, buf + sizeof(buf), v, std::chars_format::scientific);
    std::string s(buf, res.ptr);
    std::string sign;
    if (s[0] == '-') { sign = "-"; s = s.substr(1); }
    const size_t e = s.find('e');
    std::string mant = s.substr(0, e);
    const int exp10 = std::stoi(s.substr(e + 1));
    std::string digits;
    for (char c : mant)
        if (c != '.') digits += c;
    const int k = (int)digits.size(), n = exp10 + 1;
    std::string out;
    if (k <= n && n <= 15) {
        out = digits + std::string(n - k, '0') + ".0";
    } else if (0 < n && n <= 15) {
        out = digits.substr(0, n) + "." + digits.substr(n);
    } else if (-4 < n && n <= 0) {
        out = "0." + std::string(-n, '0') + digits;
    } else {
        const int x = n - 1;
        char eb[16];
        snprintf(eb, sizeof(eb), "e%c%02d", x < 0 ? '-' : '+', x < 0 ? -x : x);
        out = digits.substr(0, 1) + (k > 1 ? "." + digits.substr(1) : std::string()) + eb;
    }
    return sign + out;
}

}  // namespace fb
