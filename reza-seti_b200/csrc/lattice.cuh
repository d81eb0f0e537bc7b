// Lattice tables shared by host and device code.
//
// D3Q19 uses the reference's direction order (LatticeModel.cpp:92-192): the
// six axis directions, the twelve edge directions, and the rest direction
// last (index 18). D3Q27 uses the reference's D3Q27 order
// (LatticeModel.cpp:249-375): rest first (index 0). Keeping the reference's
// order means populations cross the C ABI without reindexing.
#pragma once

#include <cstdint>
#include <type_traits>

namespace lbm {

template <int Q>
struct Lat;

template <>
struct Lat<19> {
    static constexpr int Q = 19;
    static constexpr int REST = 18;
    __host__ __device__ static constexpr int cx(int q) {
        constexpr int t[19] = {1, -1, 0, 0, 0, 0, 1, 1, 1, 1, -1, -1, -1, -1, 0, 0, 0, 0, 0};
        return t[q];
    }
    __host__ __device__ static constexpr int cy(int q) {
        constexpr int t[19] = {0, 0, 1, -1, 0, 0, 1, -1, 0, 0, 1, -1, 0, 0, 1, 1, -1, -1, 0};
        return t[q];
    }
    __host__ __device__ static constexpr int cz(int q) {
        constexpr int t[19] = {0, 0, 0, 0, 1, -1, 0, 0, 1, -1, 0, 0, 1, -1, 1, -1, 1, -1, 0};
        return t[q];
    }
    __host__ __device__ static constexpr int opp(int q) {
        constexpr int t[19] = {1, 0, 3, 2, 5, 4, 11, 10, 13, 12, 7, 6, 9, 8, 17, 16, 15, 14, 18};
        return t[q];
    }
    // weights written as the reference writes them (2/36, 1/36, 12/36)
    __host__ __device__ static constexpr double w(int q) {
        return q < 6 ? 2.0 / 36.0 : (q < 18 ? 1.0 / 36.0 : 12.0 / 36.0);
    }
};

template <>
struct Lat<27> {
    static constexpr int Q = 27;
    static constexpr int REST = 0;
    __host__ __device__ static constexpr int cx(int q) {
        constexpr int t[27] = {0, 1, -1, 0, 0, 0, 0, 1, 1, -1, -1, 1, -1, 1,
                               -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1};
        return t[q];
    }
    __host__ __device__ static constexpr int cy(int q) {
        constexpr int t[27] = {0, 0, 0, 1, -1, 0, 0, 1, -1, 1, -1, 0, 0, 0,
                               0, 1, 1, -1, -1, 1, -1, 1, -1, -1, 1, -1, 1};
        return t[q];
    }
    __host__ __device__ static constexpr int cz(int q) {
        constexpr int t[27] = {0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, 1, -1,
                               -1, 1, -1, 1, -1, 1, -1, -1, 1, 1, -1, -1, 1};
        return t[q];
    }
    __host__ __device__ static constexpr int opp(int q) {
        constexpr int t[27] = {0, 2, 1, 4, 3, 6, 5, 10, 9, 8, 7, 14, 13, 12,
                               11, 18, 17, 16, 15, 20, 19, 22, 21, 24, 23, 26, 25};
        return t[q];
    }
    __host__ __device__ static constexpr double w(int q) {
        return q == 0 ? 8.0 / 27.0 : (q < 7 ? 2.0 / 27.0 : (q < 19 ? 1.0 / 54.0 : 1.0 / 216.0));
    }
};

// Per-node metadata word: bit q (q < Q) set when the neighbour in direction q
// exists (the rest direction's bit is always set); two bits of node kind; one
// bit marking a near-wall (wall-shear-stress) node; the remaining high bits
// hold the node's segment index relative to its block's first segment. A
// segment is a run of consecutive nodes (in the compact x-major, z-fastest
// order) whose neighbours in every direction sit at the same index offset;
// the offsets are stored once per segment, so a node costs one metadata word
// instead of a Q-entry neighbour table.
template <int Q>
struct Meta {
    using T = typename std::conditional<(Q <= 19), uint32_t, uint64_t>::type;
    static constexpr int KIND_SHIFT = Q;
    static constexpr int NW_SHIFT = Q + 2;
    static constexpr int SEG_SHIFT = Q + 3;
    static constexpr int SEG_BITS = (int)sizeof(T) * 8 - SEG_SHIFT;
    __host__ __device__ static constexpr T mask_all() { return (T(1) << Q) - 1; }
};

enum NodeKind : int { KIND_FLUID = 0, KIND_INLET = 1, KIND_OUTLET = 2, KIND_WALL = 3 };

// Nodes per thread block of the streaming kernels; segments never cross a
// block, so a block's segments are a contiguous slice of the segment table.
constexpr int BLOCK_NODES = 256;

}  // namespace lbm
