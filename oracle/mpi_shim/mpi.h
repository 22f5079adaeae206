/*
 * Stand-in for the handful of MPI calls the reference solver makes.
 *
 * TEST INFRASTRUCTURE ONLY: this header lets the unmodified reference sources
 * (Fabian2598/AMG_SchwingerModel, src/*.cpp) compile into the CPU oracle under
 * oracle/_ref/.  Nothing in the product library includes it.
 *
 * Calls used by the reference:
 *   MPI_Init / MPI_Finalize            src/main.cpp:48,176
 *   MPI_Comm_size / MPI_Comm_rank      src/sap.cpp:68-70, src/amg.cpp:5, include/amg.h:106
 *   MPI_Allreduce(DOUBLE_COMPLEX, SUM) src/sap.cpp:113,149
 *   MPI_Barrier                        src/amg.cpp:279,281, src/tests.cpp, src/main.cpp
 *   MPI_Wtime                          include/amg.h:109-111, src/tests.cpp:75-79
 *
 * One rank (the default): an all-reduce of a sum is a copy.  Each buffer entry has exactly
 * one contributor, so the result is bit-identical to an np = NB/2 run of the reference
 * provided SAPV::sap_blocks_per_proc covers every block of a colour.
 *
 * Several ranks (oracle_mpi_spawn(np, bytes), called by the harness before any work): the
 * process forks np - 1 children that run the same program as ranks 1..np-1, as mpirun would
 * start them; the reference then splits its SAP block solves among the ranks
 * (src/sap.cpp:77-78) and every rank repeats the rest, as under MPI.  Allreduce and Barrier
 * go through an anonymous shared mapping made before the fork: each rank copies its buffer
 * into its slot, each sums a 1/np share of the entries in rank order into a result buffer,
 * and every rank copies the result out, with a barrier between the steps.  The sum of one
 * contributor and exact zeros is exact, so results equal the one-rank run's (up to the sign
 * of zero entries).  Waits are bounded by liveness checks: a rank that sees another rank's
 * process gone (or its parent gone) while the barrier is open exits with an error.
 */
#ifndef ORACLE_MPI_SHIM_H
#define ORACLE_MPI_SHIM_H

#include <algorithm>
#include <atomic>
#include <csignal>
#include <new>
#include <chrono>
#include <complex>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include <sched.h>
#include <sys/mman.h>
#include <sys/wait.h>
#include <unistd.h>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;

#define MPI_COMM_WORLD 0
#define MPI_DOUBLE_COMPLEX 1
#define MPI_DOUBLE 2
#define MPI_INT 3
#define MPI_SUM 0
#define MPI_SUCCESS 0

inline int oracle_mpi_type_size(MPI_Datatype t) {
    switch (t) {
        case MPI_DOUBLE_COMPLEX: return (int)sizeof(std::complex<double>);
        case MPI_DOUBLE: return (int)sizeof(double);
        case MPI_INT: return (int)sizeof(int);
        default: return 1;
    }
}

// ---- process group -------------------------------------------------------------------
struct oracle_mpi_ctl {
    std::atomic<int> count;   // ranks arrived at the open barrier
    std::atomic<int> gen;     // barrier generation
    std::atomic<int> failed;  // 1: a rank gave up; 2: rank 0 has finished the job
};

struct oracle_mpi_state {
    int rank = 0, size = 1;
    pid_t parent = 0;
    std::vector<pid_t> kids;
    char* shm = nullptr;
    size_t slot_bytes = 0;
};

inline oracle_mpi_state& oracle_mpi() {
    static oracle_mpi_state s;
    return s;
}

constexpr size_t kOracleMpiHeader = 4096;

inline oracle_mpi_ctl* oracle_mpi_control() { return reinterpret_cast<oracle_mpi_ctl*>(oracle_mpi().shm); }
inline char* oracle_mpi_result() { return oracle_mpi().shm + kOracleMpiHeader; }
inline char* oracle_mpi_slot(int r) {
    auto& s = oracle_mpi();
    return s.shm + kOracleMpiHeader + (size_t)(r + 1) * s.slot_bytes;
}

[[noreturn]] inline void oracle_mpi_fail(const char* why) {
    auto& s = oracle_mpi();
    std::fprintf(stderr, "oracle mpi shim, rank %d: %s\n", s.rank, why);
    if (s.shm) oracle_mpi_control()->failed.store(1);
    for (pid_t k : s.kids) kill(k, SIGTERM);
    std::_Exit(70);
}

// Called while a barrier of generation g is open: gives up when a rank has failed or rank 0
// has finished (the flag counts only if this barrier is still open after it was read), when
// the parent (rank 0) is gone, or when a child rank has exited while the barrier is open.
inline void oracle_mpi_check_alive(oracle_mpi_ctl* c, int g) {
    auto& s = oracle_mpi();
    const int f = c->failed.load(std::memory_order_acquire);
    if (f != 0 && c->gen.load(std::memory_order_acquire) == g)
        oracle_mpi_fail(f == 1 ? "another rank failed" : "rank 0 finished while this rank waits in a collective");
    if (s.rank != 0 && getppid() != s.parent) oracle_mpi_fail("rank 0 is gone");
    for (pid_t k : s.kids) {
        siginfo_t info;
        info.si_pid = 0;
        if (waitid(P_PID, (id_t)k, &info, WEXITED | WNOHANG | WNOWAIT) == 0 && info.si_pid == k &&
            c->gen.load(std::memory_order_acquire) == g)
            oracle_mpi_fail("a rank exited inside a collective");
    }
}

inline void oracle_mpi_barrier() {
    auto& s = oracle_mpi();
    if (s.size == 1) return;
    oracle_mpi_ctl* c = oracle_mpi_control();
    const int g = c->gen.load(std::memory_order_acquire);
    if (c->count.fetch_add(1, std::memory_order_acq_rel) == s.size - 1) {
        c->count.store(0, std::memory_order_relaxed);
        c->gen.fetch_add(1, std::memory_order_release);
        return;
    }
    for (long spin = 1; c->gen.load(std::memory_order_acquire) == g; spin++) {
        if ((spin & 1023) == 0) {
            sched_yield();
            oracle_mpi_check_alive(c, g);
        }
    }
}

// rank 0, at exit: waits for the other ranks; a rank that failed makes the run fail
inline void oracle_mpi_join() {
    auto& s = oracle_mpi();
    if (s.rank != 0) return;
    // a rank still waiting in a collective now can never be released: let it give up
    if (s.shm) oracle_mpi_control()->failed.store(2, std::memory_order_release);
    bool ok = true;
    for (pid_t k : s.kids) {
        int st = 0;
        if (waitpid(k, &st, 0) != k || !WIFEXITED(st) || WEXITSTATUS(st) != 0) ok = false;
    }
    s.kids.clear();
    if (!ok) {
        std::fprintf(stderr, "oracle mpi shim: a rank failed\n");
        std::_Exit(71);
    }
}

// Starts np ranks of this program (the caller continues as rank 0); every rank's
// Allreduce buffer may hold up to slot_bytes bytes.
inline void oracle_mpi_spawn(int np, size_t slot_bytes) {
    auto& s = oracle_mpi();
    if (np <= 1 || s.size > 1) return;
    slot_bytes = (slot_bytes + 255) & ~(size_t)255;
    const size_t total = kOracleMpiHeader + (size_t)(np + 1) * slot_bytes;
    void* p = mmap(nullptr, total, PROT_READ | PROT_WRITE, MAP_SHARED | MAP_ANONYMOUS, -1, 0);
    if (p == MAP_FAILED) oracle_mpi_fail("mmap of the shared buffers failed");
    s.shm = static_cast<char*>(p);
    oracle_mpi_ctl* c = new (s.shm) oracle_mpi_ctl();
    c->count.store(0);
    c->gen.store(0);
    c->failed.store(0);
    s.slot_bytes = slot_bytes;
    s.size = np;
    s.parent = getpid();
    std::fflush(nullptr);
    for (int r = 1; r < np; r++) {
        const pid_t k = fork();
        if (k < 0) oracle_mpi_fail("fork failed");
        if (k == 0) {
            s.rank = r;
            s.kids.clear();
            return;
        }
        s.kids.push_back(k);
    }
    std::atexit(oracle_mpi_join);
}

inline int MPI_Init(int*, char***) { return MPI_SUCCESS; }
inline int MPI_Finalize() { return MPI_SUCCESS; }
inline int MPI_Comm_size(MPI_Comm, int* size) { *size = oracle_mpi().size; return MPI_SUCCESS; }
inline int MPI_Comm_rank(MPI_Comm, int* rank) { *rank = oracle_mpi().rank; return MPI_SUCCESS; }
inline int MPI_Barrier(MPI_Comm) {
    oracle_mpi_barrier();
    return MPI_SUCCESS;
}

inline int MPI_Allreduce(const void* sendbuf, void* recvbuf, int count, MPI_Datatype type, MPI_Op, MPI_Comm) {
    auto& s = oracle_mpi();
    const size_t bytes = (size_t)count * oracle_mpi_type_size(type);
    if (s.size == 1) {
        if (sendbuf != recvbuf) std::memcpy(recvbuf, sendbuf, bytes);
        return MPI_SUCCESS;
    }
    if (type != MPI_DOUBLE_COMPLEX && type != MPI_DOUBLE) oracle_mpi_fail("Allreduce: only sums of doubles");
    if (bytes > s.slot_bytes) oracle_mpi_fail("Allreduce: buffer larger than the shared slot");
    std::memcpy(oracle_mpi_slot(s.rank), sendbuf, bytes);
    oracle_mpi_barrier();
    const size_t n = bytes / sizeof(double);
    const size_t share = (n + s.size - 1) / s.size;
    const size_t lo = std::min(n, (size_t)s.rank * share), hi = std::min(n, lo + share);
    double* res = reinterpret_cast<double*>(oracle_mpi_result());
    for (size_t i = lo; i < hi; i++) {
        double a = reinterpret_cast<const double*>(oracle_mpi_slot(0))[i];
        for (int r = 1; r < s.size; r++) a += reinterpret_cast<const double*>(oracle_mpi_slot(r))[i];
        res[i] = a;
    }
    oracle_mpi_barrier();
    std::memcpy(recvbuf, res, bytes);
    return MPI_SUCCESS;
}

inline double MPI_Wtime() {
    using clk = std::chrono::steady_clock;
    return std::chrono::duration<double>(clk::now().time_since_epoch()).count();
}

#endif
