// Codes whose structure is compiled into the int8 decoder (columns and
// circulant shifts become immediates; no table loads in the inner loops).
//
// IEEE 802.11ad rate-1/2 base matrix (8 x 16, Z = 42), as listed in the
// standard and in the reference's matlab/LDPC/GetHMatrix.m:28-38.  Edges of a
// layer are in increasing column order, as gen_decode.m:11-16 writes them.
// A table loaded at run time matches when it has the same columns and each
// layer's shifts differ from these by one constant (mod Z): that is the
// reference's per-layer check relabel (decode_method.m:28-48), which permutes
// the checks of a layer and leaves the decoding unchanged.
#pragma once

namespace ldpc {

struct Code11ad12 {
    static constexpr int Z = 42, L = 8, MCOL = 16;
    __host__ __device__ static constexpr int maxd(int l) {
        constexpr int rw[] = {5, 6, 6, 6, 7, 7, 7, 8};
        return rw[l];
    }
    __host__ __device__ static constexpr int slot(int l, int j) {
        int b = 0;
        for (int i = 0; i < l; ++i) b += maxd(i);
        return b + j;
    }
    __host__ __device__ static constexpr int col(int e) {
        constexpr int c[] = {0, 2, 4, 6, 8,           0, 2, 4, 7, 8, 9,      1, 3, 5, 7, 9, 10,
                             1, 3, 5, 6, 10, 11,      0, 2, 4, 6, 8, 11, 12, 0, 2, 5, 7, 9, 11, 13,
                             1, 3, 5, 7, 10, 13, 14,  1, 3, 4, 6, 8, 12, 14, 15};
        return c[e];
    }
    __host__ __device__ static constexpr int shift(int e) {
        constexpr int s[] = {40, 38, 13, 5, 18,       34, 35, 27, 30, 2, 1,  36, 31, 7, 34, 10, 41,
                             27, 18, 12, 20, 15, 6,   35, 41, 40, 39, 28, 3, 28, 29, 0, 22, 4, 28, 27, 23,
                             31, 23, 21, 20, 12, 0, 13, 22, 34, 31, 14, 4, 13, 22, 24};
        return s[e];
    }
    static constexpr int E = 52;
    static constexpr int D = 8;
};

}  // namespace ldpc
