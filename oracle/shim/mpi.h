// Test infrastructure for the oracle build only.
//
// Minimal stand-in for the MPI C++ bindings (the `MPI::` namespace removed in
// MPI-3) that the reference's phase-field sources call.  Neither this
// container nor the GPU hosts ship an MPI, so the reference CPU build links
// against this header instead.
//
// Ranks are real processes: with MB_SHIM_NP=P (default 1), MPI::Init() forks
// P-1 children that share one anonymous mapping holding a process-shared
// barrier and one mailbox per rank.  That is enough for the reference's
// communication pattern, in which every rank calls the same collective
// sequence in lockstep:
//   - COMM_WORLD.Sendrecv  (SfieldFD.cpp:274,285): each rank posts its send
//     buffer in its own mailbox, all ranks meet at the barrier, and each rank
//     copies from the mailbox of its `source`;
//   - COMM_WORLD.Barrier   (every PF type, SfieldFD.cpp:397,419);
//   - COMM_WORLD.Reduce    (TIPS4.cpp:235-236), summing into `root`;
//   - Init / Finalize      (MesoExecute.cpp:19,42).
// Point-to-point messages that are not paired in lockstep are not supported.
#pragma once

#include <cstddef>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <pthread.h>
#include <sys/mman.h>
#include <sys/types.h>
#include <sys/wait.h>
#include <unistd.h>

namespace MPI {

struct Datatype {
    int bytes;
    int is_int;
};
struct Op {
    int code;
};
struct Status {};

static const Datatype DOUBLE = {8, 0};
static const Datatype INT = {4, 1};
static const Op SUM = {0};

namespace detail {

struct Shared {
    pthread_barrier_t barrier;
    size_t slot_bytes;
};

struct State {
    int rank = 0;
    int np = 1;
    Shared* shared = nullptr;
    char* slots = nullptr;
    pid_t children[1024];
    int nchildren = 0;
};

inline State& state()
{
    static State s;
    return s;
}

inline void barrier()
{
    State& s = state();
    if (s.np > 1) pthread_barrier_wait(&s.shared->barrier);
}

inline char* slot(int r)
{
    State& s = state();
    return s.slots + (size_t)r * s.shared->slot_bytes;
}

inline void fail(const char* what)
{
    std::fprintf(stderr, "mpi shim: %s\n", what);
    std::fflush(stderr);
    std::abort();
}

}  // namespace detail

inline void Init()
{
    detail::State& s = detail::state();
    const char* env = std::getenv("MB_SHIM_NP");
    int np = env ? std::atoi(env) : 1;
    if (np < 1) np = 1;
    if (np > 1024) detail::fail("MB_SHIM_NP above 1024");
    s.np = np;
    s.rank = 0;
    if (np == 1) return;

    const char* slot_env = std::getenv("MB_SHIM_SLOT_MB");
    size_t slot_bytes = (size_t)(slot_env ? std::atoll(slot_env) : 64) << 20;
    size_t total = sizeof(detail::Shared) + 64 + (size_t)np * slot_bytes;
    void* mem = mmap(nullptr, total, PROT_READ | PROT_WRITE,
                     MAP_SHARED | MAP_ANONYMOUS | MAP_NORESERVE, -1, 0);
    if (mem == MAP_FAILED) detail::fail("mmap of the shared mailboxes failed");
    s.shared = static_cast<detail::Shared*>(mem);
    s.shared->slot_bytes = slot_bytes;
    s.slots = static_cast<char*>(mem) + ((sizeof(detail::Shared) + 63) / 64) * 64;

    pthread_barrierattr_t attr;
    pthread_barrierattr_init(&attr);
    pthread_barrierattr_setpshared(&attr, PTHREAD_PROCESS_SHARED);
    pthread_barrier_init(&s.shared->barrier, &attr, (unsigned)np);
    pthread_barrierattr_destroy(&attr);

    std::fflush(nullptr);  // children must not re-flush the parent's buffers
    for (int r = 1; r < np; ++r) {
        pid_t pid = fork();
        if (pid < 0) detail::fail("fork failed");
        if (pid == 0) {
            s.rank = r;
            s.nchildren = 0;
            return;
        }
        s.children[s.nchildren++] = pid;
    }
}

inline void Finalize()
{
    detail::State& s = detail::state();
    if (s.np == 1) return;
    detail::barrier();
    if (s.rank != 0) {
        std::fflush(nullptr);
        _exit(0);
    }
    for (int i = 0; i < s.nchildren; ++i) {
        int status = 0;
        waitpid(s.children[i], &status, 0);
    }
}

struct Intracomm {
    int Get_rank() const { return detail::state().rank; }
    int Get_size() const { return detail::state().np; }
    void Barrier() const { detail::barrier(); }

    void Sendrecv(const void* sendbuf, int sendcount, const Datatype& sendtype, int /*dest*/,
                  int /*sendtag*/, void* recvbuf, int recvcount, const Datatype& recvtype,
                  int source, int /*recvtag*/, Status& /*status*/) const
    {
        detail::State& s = detail::state();
        size_t sbytes = (size_t)sendcount * sendtype.bytes;
        size_t rbytes = (size_t)recvcount * recvtype.bytes;
        if (s.np == 1) {
            std::memmove(recvbuf, sendbuf, rbytes < sbytes ? rbytes : sbytes);
            return;
        }
        if (sbytes > s.shared->slot_bytes) detail::fail("message larger than MB_SHIM_SLOT_MB");
        std::memcpy(detail::slot(s.rank), sendbuf, sbytes);
        detail::barrier();
        std::memcpy(recvbuf, detail::slot(source), rbytes);
        detail::barrier();
    }

    void Reduce(const void* sendbuf, void* recvbuf, int count, const Datatype& type,
                const Op& /*op: only SUM is used*/, int root) const
    {
        detail::State& s = detail::state();
        size_t bytes = (size_t)count * type.bytes;
        if (s.np == 1) {
            std::memmove(recvbuf, sendbuf, bytes);
            return;
        }
        if (bytes > s.shared->slot_bytes) detail::fail("message larger than MB_SHIM_SLOT_MB");
        std::memcpy(detail::slot(s.rank), sendbuf, bytes);
        detail::barrier();
        if (s.rank == root) {
            for (int i = 0; i < count; ++i) {
                if (type.is_int) {
                    int acc = 0;
                    for (int r = 0; r < s.np; ++r) acc += reinterpret_cast<const int*>(detail::slot(r))[i];
                    static_cast<int*>(recvbuf)[i] = acc;
                } else {
                    double acc = 0.0;
                    for (int r = 0; r < s.np; ++r) acc += reinterpret_cast<const double*>(detail::slot(r))[i];
                    static_cast<double*>(recvbuf)[i] = acc;
                }
            }
        }
        detail::barrier();
    }
};

static Intracomm COMM_WORLD;

}  // namespace MPI

typedef int MPI_Comm;
#define MPI_COMM_WORLD 0
#define MPI_INT (MPI::INT)
#define MPI_DOUBLE (MPI::DOUBLE)
#define MPI_SUM (MPI::SUM)
