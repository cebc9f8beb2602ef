// Test-only harness around the reference's UNMODIFIED CPU orienters in
// MST.cpp (orient_kruskal, MST.cpp:399-423; orient, :426-447), compiled from
// the reference's own source by oracle/ref/Makefile into
// oracle/_ref/libegtref_mst.so.  The reference functions print progress to
// std::cout; the harness sends that output to a null buffer for the duration
// of the call.  Nothing in the product links or loads this library.
#include <chrono>
#include <iostream>
#include <streambuf>

#include "MST.h"

namespace {
struct NullBuf : std::streambuf {
    int overflow(int c) override { return c; }
};
}  // namespace

extern "C" {

// orient_kruskal(knn, nx, ny, nz, x, y, z, N, k, k_use) on host arrays, in
// place; returns the call's wall time in milliseconds.
double egtref_orient_kruskal(int* knn, float* nx, float* ny, float* nz, float* x, float* y, float* z, int n, int k,
                             int k_use) {
    NullBuf nb;
    std::streambuf* old = std::cout.rdbuf(&nb);
    const auto t0 = std::chrono::steady_clock::now();
    orient_kruskal(knn, nx, ny, nz, x, y, z, n, k, k_use);
    const auto t1 = std::chrono::steady_clock::now();
    std::cout.rdbuf(old);
    return std::chrono::duration<double, std::milli>(t1 - t0).count();
}

}  // extern "C"
