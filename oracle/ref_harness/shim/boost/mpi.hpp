// Single-rank stand-in for the Boost.MPI API surface milupHPC's hot-path
// sources use; it lets those sources compile unmodified for one process.
// Test infrastructure only (oracle/ref_harness).
#pragma once
#include <chrono>
#include <functional>
#include <vector>

#include "../mpi.h"

namespace boost {
namespace serialization {
class access {};
}  // namespace serialization
namespace mpi {
struct status {};
struct request {
    status wait() { return status(); }
    bool test() { return true; }
};
template <class It>
void wait_all(It, It) {}
struct environment {
    environment() {}
    environment(int&, char**&) {}
};
// point-to-point calls never happen with one rank
struct communicator {
    int rank() const { return 0; }
    int size() const { return 1; }
    void barrier() const {}
    template <class... A>
    request isend(A&&...) const { return request(); }
    template <class... A>
    request irecv(A&&...) const { return request(); }
    template <class... A>
    void send(A&&...) const {}
    template <class... A>
    status recv(A&&...) const { return status(); }
};
template <class T>
struct inplace_t {
    T buf;
    explicit inplace_t(T b) : buf(b) {}
};
template <class T>
inplace_t<T> inplace(T b) { return inplace_t<T>(b); }
template <class T>
struct minimum {
    T operator()(const T& a, const T& b) const { return a < b ? a : b; }
};
template <class T>
struct maximum {
    T operator()(const T& a, const T& b) const { return a < b ? b : a; }
};
// one rank: every reduction is the identity
template <class T, class Op>
void all_reduce(const communicator&, inplace_t<T>, int, Op) {}
template <class T, class Op>
void all_reduce(const communicator&, inplace_t<T>, Op) {}
template <class T, class Op>
void all_reduce(const communicator&, const T& in, T& out, Op) { out = in; }
template <class T, class Op>
void all_reduce(const communicator&, const T* in, int n, T* out, Op) {
    for (int i = 0; i < n; ++i) out[i] = in[i];
}
template <class... A>
void broadcast(A&&...) {}
class timer {
    std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();
public:
    void restart() { t0 = std::chrono::steady_clock::now(); }
    double elapsed() const {
        return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    }
};
}  // namespace mpi
}  // namespace boost
