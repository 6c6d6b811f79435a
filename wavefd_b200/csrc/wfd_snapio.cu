// Snapshot files: saved forward wavefields on disk with an offsets/lengths index, the role of
// Compressor / compressedwrite / compressedread! (compressedio.jl:1-137) for the plain FP32 fallback
// of Born imaging (and for codec payloads). As there, field i of a file is written once and read
// back in any order; a short write is an error naming the bytes written and the file.
//
// Format (little-endian), all offsets in bytes from the start of the file:
//   [0, hdr)                header: "WFDSNAP1", u32 version (1), u32 flags, i64 nfields,
//                           i64 slot, i64 data offset (= hdr), then per field i64 offset and
//                           i64 length (-1 = never written); hdr is a multiple of 4096
//   hdr + i * slot          field i's payload; slot = the largest payload rounded up to 4096
// The header is written by WFD_Snap_Sync and WFD_Snap_Close; fixed slots let fields be written in
// any order and read at a computed offset, and keep every payload 4096-aligned for O_DIRECT.
//
// Device payloads (the default) never hold up the caller's stream for the host link: a write copies
// the array into a device staging slot on the caller's stream (so the caller may overwrite it right
// after), then to pinned host memory on the file's copy stream, and a worker thread pwrite()s it; a
// read (or a prefetch, which starts the same work early) has the worker pread() into pinned memory
// and copy to a device staging slot on the copy stream, and the read itself is a device-to-device
// copy on the caller's stream behind an event. Host payloads (WFD_SNAP_HOST) go straight through
// pwrite()/pread() and make no CUDA call.
#include <cuda_runtime.h>
#include <fcntl.h>
#include <unistd.h>

#include <cerrno>
#include <chrono>
#include <condition_variable>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "wavefd_b200.h"
#include "wfd_alloc.h"
#include "wfd_prop.h"

namespace wfd {
namespace snap {

constexpr char kMagic[8] = {'W', 'F', 'D', 'S', 'N', 'A', 'P', '1'};
constexpr uint32_t kVersion = 1;
constexpr long kAlign = 4096;
constexpr int kStages = 3;
constexpr auto kWaitLimit = std::chrono::seconds(600);  // a host wait for the worker gives up after this

long round_up(long v, long a) { return (v + a - 1) / a * a; }
long header_bytes(long nfields) { return round_up(48 + 16 * nfields, kAlign); }

enum class St { FREE, WRITE, READ, READY };

struct Stage {
    void *host = nullptr;  // pinned
    void *dev = nullptr;
    St st = St::FREE;
    long field = -1, nbytes = 0;
    cudaEvent_t host_ev = nullptr;      // the last GPU copy touching `host` is done after this
    cudaEvent_t dev_free_ev = nullptr;  // the last GPU use of `dev` is done after this
    cudaEvent_t staged_ev = nullptr;    // a write's device-to-device copy is done after this
    bool host_ev_set = false, dev_free_set = false;
};

struct Job {
    bool write;
    int stage;
};

struct File {
    std::string path;
    int fd = -1;
    bool host_mode = false, readonly = false, direct = false;
    uint32_t flags = 0;
    long nfields = 0, slot = 0, hdr = 0;
    std::vector<long> len;
    int device = 0;
    cudaStream_t copy = nullptr;
    Stage stage[kStages];
    std::thread worker;
    std::mutex mu;
    std::condition_variable cv_job, cv_done;
    std::deque<Job> jobs;
    bool stop = false;
    int status = WFD_OK;
    std::string message;
};

// I/O, CUDA and time-limit errors stay with the file (every later call returns them); a bad
// argument only fails its own call
int fail(File *f, int code, const std::string &msg) {
    if (f && code != WFD_ERR_ARG) {
        std::lock_guard<std::mutex> lk(f->mu);
        if (f->status == WFD_OK) {
            f->status = code;
            f->message = msg;
        }
    }
    set_global_error(code, msg);
    return code;
}

int cuda_fail(File *f, cudaError_t e, const char *what) {
    return fail(f, WFD_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

// pwrite/pread of a whole range (they may transfer less than asked)
long write_all(int fd, const void *buf, long n, long off) {
    long done = 0;
    while (done < n) {
        const ssize_t r = pwrite(fd, static_cast<const char *>(buf) + done, (size_t)(n - done), off + done);
        if (r < 0 && errno == EINTR) continue;
        if (r <= 0) break;
        done += r;
    }
    return done;
}
long read_all(int fd, void *buf, long n, long off) {
    long done = 0;
    while (done < n) {
        const ssize_t r = pread(fd, static_cast<char *>(buf) + done, (size_t)(n - done), off + done);
        if (r < 0 && errno == EINTR) continue;
        if (r <= 0) break;
        done += r;
    }
    return done;
}

std::string io_message(const File *f, const char *verb, long done, long n, long field) {
    const int e = errno;
    return std::string(verb) + " " + std::to_string(done) + " of " + std::to_string(n) + " bytes of field " +
           std::to_string(field) + " in " + f->path + (e ? std::string(": ") + std::strerror(e) : std::string());
}

int write_header(File *f) {
    void *mem = nullptr;  // page-aligned, as O_DIRECT requires
    if (posix_memalign(&mem, kAlign, (size_t)f->hdr) != 0) return fail(f, WFD_ERR_ALLOC, "WFD_Snap: header buffer");
    char *h = static_cast<char *>(mem);
    std::memset(h, 0, (size_t)f->hdr);
    std::memcpy(h, kMagic, 8);
    std::memcpy(h + 8, &kVersion, 4);
    std::memcpy(h + 12, &f->flags, 4);
    const int64_t v[3] = {f->nfields, f->slot, f->hdr};
    std::memcpy(h + 16, v, sizeof v);
    {
        std::lock_guard<std::mutex> lk(f->mu);
        for (long i = 0; i < f->nfields; i++) {
            const int64_t e[2] = {f->hdr + i * f->slot, f->len[i]};
            std::memcpy(h + 48 + 16 * i, e, sizeof e);
        }
    }
    errno = 0;
    const long done = write_all(f->fd, h, f->hdr, 0);
    free(mem);
    if (done != f->hdr) return fail(f, WFD_ERR_IO, io_message(f, "wrote", done, f->hdr, -1) + " (header)");
    return WFD_OK;
}

// payload bytes actually transferred: with O_DIRECT the whole 4096-aligned span
long io_bytes(const File *f, long n) { return f->direct ? round_up(n, kAlign) : n; }

void worker_main(File *f) {
    cudaSetDevice(f->device);
    for (;;) {
        Job job;
        {
            std::unique_lock<std::mutex> lk(f->mu);
            f->cv_job.wait(lk, [&] { return f->stop || !f->jobs.empty(); });
            if (f->jobs.empty()) return;  // stop with nothing left
            job = f->jobs.front();
            f->jobs.pop_front();
        }
        Stage &s = f->stage[job.stage];
        if (job.write) {
            // the pinned copy has landed once the D2H copy is done
            cudaError_t e = cudaEventSynchronize(s.host_ev);
            if (e != cudaSuccess) cuda_fail(f, e, "WFD_Snap_Write (copy to host)");
            else {
                errno = 0;
                const long n = io_bytes(f, s.nbytes);
                const long done = write_all(f->fd, s.host, n, f->hdr + s.field * f->slot);
                if (done != n) fail(f, WFD_ERR_IO, io_message(f, "wrote", done, n, s.field));
                else {
                    std::lock_guard<std::mutex> lk(f->mu);
                    f->len[s.field] = s.nbytes;
                }
            }
            std::lock_guard<std::mutex> lk(f->mu);
            s.st = St::FREE;
            s.field = -1;
        } else {
            // the pinned buffer's previous H2D copy must be done before pread overwrites it
            cudaError_t e = s.host_ev_set ? cudaEventSynchronize(s.host_ev) : cudaSuccess;
            bool ok = e == cudaSuccess;
            if (!ok) cuda_fail(f, e, "WFD_Snap_Read (previous copy)");
            if (ok) {
                errno = 0;
                const long n = io_bytes(f, s.nbytes);
                const long done = read_all(f->fd, s.host, n, f->hdr + s.field * f->slot);
                if (done < s.nbytes) {
                    fail(f, WFD_ERR_IO, io_message(f, "read", done, s.nbytes, s.field));
                    ok = false;
                }
            }
            if (ok && s.dev_free_set) ok = (e = cudaStreamWaitEvent(f->copy, s.dev_free_ev, 0)) == cudaSuccess;
            if (ok) ok = (e = cudaMemcpyAsync(s.dev, s.host, s.nbytes, cudaMemcpyHostToDevice, f->copy)) == cudaSuccess;
            if (ok) ok = (e = cudaEventRecord(s.host_ev, f->copy)) == cudaSuccess;
            if (!ok && e != cudaSuccess) cuda_fail(f, e, "WFD_Snap_Read (copy to device)");
            std::lock_guard<std::mutex> lk(f->mu);
            s.host_ev_set = ok;
            if (ok) s.st = St::READY;
            else {
                s.st = St::FREE;
                s.field = -1;
            }
        }
        f->cv_done.notify_all();
    }
}

// a stage to reuse (lock held): a FREE one, else one holding a prefetched field nobody has read
// (dropped); waits for the worker when every stage has a transfer in flight
int acquire(File *f, std::unique_lock<std::mutex> &lk) {
    auto pick = [&]() {
        for (int i = 0; i < kStages; i++)
            if (f->stage[i].st == St::FREE) return i;
        for (int i = 0; i < kStages; i++)
            if (f->stage[i].st == St::READY) {
                f->stage[i].st = St::FREE;
                f->stage[i].field = -1;
                return i;
            }
        return -1;
    };
    int s = pick();
    if (s >= 0) return s;
    if (!f->cv_done.wait_for(lk, kWaitLimit, [&] {
            for (int i = 0; i < kStages; i++)
                if (f->stage[i].st == St::FREE || f->stage[i].st == St::READY) return true;
            return false;
        }))
        return -1;
    return pick();
}

int find(File *f, long field, St a, St b) {
    for (int i = 0; i < kStages; i++)
        if (f->stage[i].field == field && (f->stage[i].st == a || f->stage[i].st == b)) return i;
    return -1;
}

bool pending_write(File *f, long field) { return find(f, field, St::WRITE, St::WRITE) >= 0; }

int check(File *f) {
    std::lock_guard<std::mutex> lk(f->mu);
    return f->status;
}

// start reading field i into a stage (lock held); returns the stage or -1
int start_read(File *f, long i, std::unique_lock<std::mutex> &lk) {
    int s = find(f, i, St::READ, St::READY);
    if (s >= 0) return s;
    if (!f->cv_done.wait_for(lk, kWaitLimit, [&] { return !pending_write(f, i); })) return -1;
    if (f->len[i] < 0) return -2;
    s = acquire(f, lk);
    if (s < 0) return -1;
    Stage &st = f->stage[s];
    st.st = St::READ;
    st.field = i;
    st.nbytes = f->len[i];
    f->jobs.push_back({false, s});
    f->cv_job.notify_one();
    return s;
}

void destroy(File *f) {
    if (!f) return;
    if (f->worker.joinable()) {
        {
            std::lock_guard<std::mutex> lk(f->mu);
            f->stop = true;
        }
        f->cv_job.notify_all();
        f->worker.join();
    }
    if (!f->host_mode) {
        for (auto &s : f->stage) {
            if (s.host) cudaFreeHost(s.host);
            if (s.dev) cudaFree(s.dev);
            if (s.host_ev) cudaEventDestroy(s.host_ev);
            if (s.dev_free_ev) cudaEventDestroy(s.dev_free_ev);
            if (s.staged_ev) cudaEventDestroy(s.staged_ev);
        }
        if (f->copy) cudaStreamDestroy(f->copy);
    }
    if (f->fd >= 0) close(f->fd);
    delete f;
}

}  // namespace snap
}  // namespace wfd

using wfd::snap::File;

extern "C" void *WFD_Snap_Open(const char *path, long nfields, long max_bytes, int flags) {
    using namespace wfd::snap;
    if (!path) {
        wfd::set_global_error(WFD_ERR_ARG, "WFD_Snap_Open: null path");
        return nullptr;
    }
    File *f = new File;
    f->path = path;
    f->host_mode = (flags & WFD_SNAP_HOST) != 0;
    f->readonly = (flags & WFD_SNAP_READ) != 0;
    f->direct = (flags & WFD_SNAP_DIRECT) != 0 && !f->host_mode;
    if (f->readonly) {
        f->fd = open(path, O_RDONLY);  // the header is read through the page cache
        if (f->fd < 0) {
            wfd::set_global_error(WFD_ERR_IO, std::string("WFD_Snap_Open: cannot open ") + path + ": " +
                                                  std::strerror(errno));
            destroy(f);
            return nullptr;
        }
        char h[48];
        if (read_all(f->fd, h, 48, 0) != 48 || std::memcmp(h, kMagic, 8) != 0) {
            wfd::set_global_error(WFD_ERR_ARG, std::string("WFD_Snap_Open: not a snapshot file: ") + path);
            destroy(f);
            return nullptr;
        }
        uint32_t ver;
        int64_t v[3];
        std::memcpy(&ver, h + 8, 4);
        std::memcpy(&f->flags, h + 12, 4);
        std::memcpy(v, h + 16, sizeof v);
        f->nfields = v[0];
        f->slot = v[1];
        f->hdr = v[2];
        if (ver != kVersion || f->nfields < 1 || f->slot < 1 || f->hdr != header_bytes(f->nfields)) {
            wfd::set_global_error(WFD_ERR_ARG, std::string("WFD_Snap_Open: unsupported header in ") + path);
            destroy(f);
            return nullptr;
        }
        std::vector<int64_t> idx((size_t)(2 * f->nfields));
        if (read_all(f->fd, idx.data(), 16 * f->nfields, 48) != 16 * f->nfields) {
            wfd::set_global_error(WFD_ERR_IO, std::string("WFD_Snap_Open: short index in ") + path);
            destroy(f);
            return nullptr;
        }
        f->len.resize((size_t)f->nfields);
        for (long i = 0; i < f->nfields; i++) f->len[i] = idx[2 * i + 1];
        if (f->direct) {  // payloads bypass the page cache; buffered if the file system refuses
            const int fd = open(path, O_RDONLY | O_DIRECT);
            if (fd >= 0) {
                close(f->fd);
                f->fd = fd;
            } else {
                f->direct = false;
            }
        }
    } else {
        if (nfields < 1 || max_bytes < 1) {
            wfd::set_global_error(WFD_ERR_ARG, "WFD_Snap_Open: nfields and max_bytes must be positive");
            destroy(f);
            return nullptr;
        }
        const int oflags = O_RDWR | O_CREAT | O_TRUNC;
        f->fd = open(path, oflags | (f->direct ? O_DIRECT : 0), 0644);
        if (f->fd < 0 && f->direct) {
            f->direct = false;
            f->fd = open(path, oflags, 0644);
        }
        if (f->fd < 0) {
            wfd::set_global_error(WFD_ERR_IO, std::string("WFD_Snap_Open: cannot create ") + path + ": " +
                                                  std::strerror(errno));
            destroy(f);
            return nullptr;
        }
        f->nfields = nfields;
        f->slot = round_up(max_bytes, kAlign);
        f->hdr = header_bytes(nfields);
        f->flags = (uint32_t)(flags & WFD_SNAP_CODEC);
        f->len.assign((size_t)nfields, -1);
    }
    if (!f->host_mode) {
        cudaError_t e = cudaGetDevice(&f->device);
        if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&f->copy, cudaStreamNonBlocking);
        for (auto &s : f->stage) {
            if (e == cudaSuccess) e = cudaHostAlloc(&s.host, (size_t)f->slot, cudaHostAllocDefault);
            if (e == cudaSuccess) e = wfd::dMalloc(&s.dev, (size_t)f->slot);
            if (e == cudaSuccess) e = cudaEventCreateWithFlags(&s.host_ev, cudaEventDisableTiming);
            if (e == cudaSuccess) e = cudaEventCreateWithFlags(&s.dev_free_ev, cudaEventDisableTiming);
            if (e == cudaSuccess) e = cudaEventCreateWithFlags(&s.staged_ev, cudaEventDisableTiming);
        }
        if (e != cudaSuccess) {
            wfd::set_global_error(e == cudaErrorMemoryAllocation ? WFD_ERR_ALLOC : WFD_ERR_CUDA,
                                  std::string("WFD_Snap_Open: ") + cudaGetErrorString(e));
            destroy(f);
            return nullptr;
        }
        f->worker = std::thread(worker_main, f);
    }
    return f;
}

extern "C" int WFD_Snap_Write(void *fp, long ifield, const void *src, long nbytes, void *stream) {
    using namespace wfd::snap;
    File *f = static_cast<File *>(fp);
    if (!f || !src || f->readonly || ifield < 0 || ifield >= f->nfields || nbytes < 1 || nbytes > f->slot)
        return fail(f, WFD_ERR_ARG, "WFD_Snap_Write: bad arguments");
    if (int st = check(f)) return st;
    if (f->host_mode) {
        const long n = nbytes;
        errno = 0;
        const long done = write_all(f->fd, src, n, f->hdr + ifield * f->slot);
        if (done != n) return fail(f, WFD_ERR_IO, io_message(f, "wrote", done, n, ifield));
        std::lock_guard<std::mutex> lk(f->mu);
        f->len[ifield] = nbytes;
        return WFD_OK;
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    std::unique_lock<std::mutex> lk(f->mu);
    // a staged read of this field is stale now
    for (auto &s : f->stage)
        if (s.field == ifield && s.st == St::READY) {
            s.st = St::FREE;
            s.field = -1;
        }
    const int si = acquire(f, lk);
    if (si < 0) {
        lk.unlock();
        return fail(f, WFD_ERR_TIMEOUT, "WFD_Snap_Write: no staging slot freed within the time limit");
    }
    Stage &s = f->stage[si];
    // caller's stream: (previous use of the device slot done) -> copy into the slot; copy stream:
    // (slot filled, previous use of the pinned buffer done) -> copy to the pinned buffer
    // (host_ev also covers a copy into the device slot of a prefetched field that was dropped)
    cudaError_t e = cudaSuccess;
    if (s.dev_free_set) e = cudaStreamWaitEvent(st, s.dev_free_ev, 0);
    if (e == cudaSuccess && s.host_ev_set) e = cudaStreamWaitEvent(st, s.host_ev, 0);
    if (e == cudaSuccess) e = cudaMemcpyAsync(s.dev, src, (size_t)nbytes, cudaMemcpyDefault, st);
    if (e == cudaSuccess) e = cudaEventRecord(s.staged_ev, st);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(f->copy, s.staged_ev, 0);
    if (e == cudaSuccess && s.host_ev_set) e = cudaStreamWaitEvent(f->copy, s.host_ev, 0);
    if (e == cudaSuccess) e = cudaMemcpyAsync(s.host, s.dev, (size_t)nbytes, cudaMemcpyDeviceToHost, f->copy);
    if (e == cudaSuccess) e = cudaEventRecord(s.host_ev, f->copy);      // the worker waits for this
    if (e == cudaSuccess) e = cudaEventRecord(s.dev_free_ev, f->copy);  // the device slot is free after it
    if (e != cudaSuccess) {
        lk.unlock();
        return cuda_fail(f, e, "WFD_Snap_Write");
    }
    s.dev_free_set = true;
    s.host_ev_set = true;
    s.st = St::WRITE;
    s.field = ifield;
    s.nbytes = nbytes;
    f->jobs.push_back({true, si});
    f->cv_job.notify_one();
    return WFD_OK;
}

extern "C" int WFD_Snap_Prefetch(void *fp, long ifield) {
    using namespace wfd::snap;
    File *f = static_cast<File *>(fp);
    if (!f || ifield < 0 || ifield >= f->nfields) return fail(f, WFD_ERR_ARG, "WFD_Snap_Prefetch: bad arguments");
    if (int st = check(f)) return st;
    if (f->host_mode) return WFD_OK;
    std::unique_lock<std::mutex> lk(f->mu);
    const int s = start_read(f, ifield, lk);
    lk.unlock();
    if (s == -2) return fail(f, WFD_ERR_ARG, "WFD_Snap_Prefetch: field " + std::to_string(ifield) + " was never written");
    if (s < 0) return fail(f, WFD_ERR_TIMEOUT, "WFD_Snap_Prefetch: no staging slot freed within the time limit");
    return WFD_OK;
}

extern "C" int WFD_Snap_Read(void *fp, long ifield, void *dst, long nbytes, void *stream) {
    using namespace wfd::snap;
    File *f = static_cast<File *>(fp);
    if (!f || !dst || ifield < 0 || ifield >= f->nfields || nbytes < 1)
        return fail(f, WFD_ERR_ARG, "WFD_Snap_Read: bad arguments");
    if (int st = check(f)) return st;
    if (f->host_mode) {
        const long n = f->len[ifield];
        if (n < 0 || n > nbytes)
            return fail(f, WFD_ERR_ARG, "WFD_Snap_Read: field " + std::to_string(ifield) +
                                            (n < 0 ? " was never written" : " is larger than the buffer"));
        errno = 0;
        const long done = read_all(f->fd, dst, n, f->hdr + ifield * f->slot);
        if (done != n) return fail(f, WFD_ERR_IO, io_message(f, "read", done, n, ifield));
        return WFD_OK;
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    std::unique_lock<std::mutex> lk(f->mu);
    if (f->len[ifield] > nbytes && !pending_write(f, ifield)) {
        lk.unlock();
        return fail(f, WFD_ERR_ARG, "WFD_Snap_Read: field " + std::to_string(ifield) + " is larger than the buffer");
    }
    const int si = start_read(f, ifield, lk);
    if (si < 0) {
        lk.unlock();
        if (si == -2) return fail(f, WFD_ERR_ARG, "WFD_Snap_Read: field " + std::to_string(ifield) + " was never written");
        return fail(f, WFD_ERR_TIMEOUT, "WFD_Snap_Read: no staging slot freed within the time limit");
    }
    Stage &s = f->stage[si];
    if (!f->cv_done.wait_for(lk, kWaitLimit, [&] { return s.st != St::READ || f->status != WFD_OK; })) {
        lk.unlock();
        return fail(f, WFD_ERR_TIMEOUT, "WFD_Snap_Read: the read did not finish within the time limit");
    }
    if (f->status != WFD_OK || s.st != St::READY || s.field != ifield) {
        const int code = f->status != WFD_OK ? f->status : WFD_ERR_IO;
        lk.unlock();
        return code == WFD_OK ? fail(f, WFD_ERR_IO, "WFD_Snap_Read: staging lost") : code;
    }
    if (s.nbytes > nbytes) {
        lk.unlock();
        return fail(f, WFD_ERR_ARG, "WFD_Snap_Read: field " + std::to_string(ifield) + " is larger than the buffer");
    }
    cudaError_t e = cudaStreamWaitEvent(st, s.host_ev, 0);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dst, s.dev, (size_t)s.nbytes, cudaMemcpyDefault, st);
    if (e == cudaSuccess) e = cudaEventRecord(s.dev_free_ev, st);
    if (e != cudaSuccess) {
        lk.unlock();
        return cuda_fail(f, e, "WFD_Snap_Read");
    }
    s.dev_free_set = true;
    s.st = St::FREE;
    s.field = -1;
    f->cv_done.notify_all();
    return WFD_OK;
}

extern "C" long WFD_Snap_Length(void *fp, long ifield) {
    using namespace wfd::snap;
    File *f = static_cast<File *>(fp);
    if (!f || ifield < 0 || ifield >= f->nfields) return -1;
    std::unique_lock<std::mutex> lk(f->mu);
    f->cv_done.wait_for(lk, kWaitLimit, [&] { return !pending_write(f, ifield); });
    return f->len[ifield];
}

extern "C" long WFD_Snap_NumFields(void *fp) { return fp ? static_cast<File *>(fp)->nfields : -1; }

extern "C" int WFD_Snap_Flags(void *fp) { return fp ? (int)static_cast<File *>(fp)->flags : -1; }

extern "C" int WFD_Snap_Sync(void *fp) {
    using namespace wfd::snap;
    File *f = static_cast<File *>(fp);
    if (!f) return WFD_ERR_ARG;
    {
        std::unique_lock<std::mutex> lk(f->mu);
        if (!f->cv_done.wait_for(lk, kWaitLimit, [&] {
                for (auto &s : f->stage)
                    if (s.st == St::WRITE || s.st == St::READ) return false;
                return true;
            })) {
            lk.unlock();
            return fail(f, WFD_ERR_TIMEOUT, "WFD_Snap_Sync: transfers did not finish within the time limit");
        }
    }
    if (int st = check(f)) return st;
    if (f->readonly) return WFD_OK;
    return write_header(f);
}

extern "C" int WFD_Snap_Close(void *fp) {
    using namespace wfd::snap;
    File *f = static_cast<File *>(fp);
    if (!f) return WFD_ERR_ARG;
    const int st = WFD_Snap_Sync(f);
    destroy(f);
    return st;
}
