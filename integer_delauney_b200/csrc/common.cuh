// Shared infrastructure for the integer Delaunay CUDA library: status codes,
// the thread-local error message, CUDA call checking and small device helpers.
//
// Error convention (mirrors the reference's, src/cuda/cuda_check.cuh:12-62):
// a failing CUDA call is reported as "<file>:<line>: <expr> failed: <msg>"
// after draining the sticky last error, and surfaces as RuntimeError at the
// Python boundary; input validation failures surface as ValueError.  Here the
// C ABI returns a status code instead of throwing, and the message is kept in
// a thread-local buffer readable through idl_last_error().
#pragma once

#include <cuda_runtime.h>
#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <stdexcept>
#include <string>

#include "../../include/idelaunay.h"

namespace idl {

// Thrown inside the library, converted to a status code at the C boundary.
struct Error : public std::runtime_error {
    int status;
    Error(int s, const std::string& m) : std::runtime_error(m), status(s) {}
};

void set_last_error(const char* msg);

inline void cuda_check(cudaError_t err, const char* expr, const char* file, int line)
{
    if (err != cudaSuccess) {
        cudaGetLastError();   // drain the sticky error so it is scoped to this call
        const char* base = std::strrchr(file, '/');
        throw Error(IDL_ERR_CUDA, std::string(base ? base + 1 : file) + ":" + std::to_string(line) +
                                      ": " + expr + " failed: " + cudaGetErrorString(err));
    }
}

[[noreturn]] inline void invalid(const std::string& msg) { throw Error(IDL_ERR_INVALID, msg); }

}  // namespace idl

namespace idl {
// Kernels this library has launched in this process (idl_launch_count()).
void count_launch();
// Device and pinned host allocations this library has made in this process
// (idl_alloc_count()).
void count_alloc();
}  // namespace idl

#define IDL_CUDA(expr) ::idl::cuda_check((expr), #expr, __FILE__, __LINE__)
#define IDL_LAUNCH()                                                            \
    do {                                                                        \
        ::idl::count_launch();                                                  \
        ::idl::cuda_check(cudaGetLastError(), "kernel launch", __FILE__, __LINE__); \
    } while (0)

// Convert exceptions into status codes at every extern "C" entry point.
#define IDL_API_BEGIN try {
#define IDL_API_END                                                  \
    }                                                                \
    catch (const ::idl::Error& e) {                                  \
        ::idl::set_last_error(e.what());                             \
        return e.status;                                             \
    }                                                                \
    catch (const std::bad_alloc&) {                                  \
        ::idl::set_last_error("host allocation failed");            \
        return IDL_ERR_CUDA;                                         \
    }                                                                \
    catch (const std::exception& e) {                                \
        ::idl::set_last_error(e.what());                             \
        return IDL_ERR_INTERNAL;                                     \
    }                                                                \
    return IDL_OK;

namespace idl {

// Label values on the Voronoi canvas.
constexpr int32_t UNDEF = -1;          // cell no seed owns yet (voronoi.cuh:14-24)
constexpr int32_t NO_TRIANGLE = -1;    // pixel no triangle contains (triangulation.cuh:14-22)

// Seeds addressable by the packed 63-bit triangle key (21 bits per id), the
// same packing the reference's registry uses (delaunay.cuh:372-374).
constexpr int64_t MAX_SEEDS = (int64_t(1) << 21) - 1;

// Largest padded canvas side.  Squared distances are int32 in the reference
// (reference/voronoi.py:30-31); 32767 keeps dx^2 + dy^2 below 2^31 and lets a
// seed position pack into 16 + 16 bits.
constexpr int MAX_CANVAS_SIDE = 32767;

__host__ __device__ inline uint32_t pack_pos(int x, int y) { return uint32_t(x) | (uint32_t(y) << 16); }
__host__ __device__ inline int pos_x(uint32_t p) { return int(p & 0xFFFFu); }
__host__ __device__ inline int pos_y(uint32_t p) { return int(p >> 16); }

__device__ __forceinline__ int32_t dist2(int x, int y, uint32_t p)
{
    const int32_t dx = x - pos_x(p), dy = y - pos_y(p);
    return dx * dx + dy * dy;
}

inline int ceil_div(int64_t a, int64_t b) { return int((a + b - 1) / b); }

inline int64_t next_pow2(int64_t v)
{
    int64_t p = 1;
    while (p < v) p <<= 1;
    return p;
}

}  // namespace idl
