// Hard decisions and error counting of one finished codeword by one warp
// (LDPC_count_errors, src/Top/LDPC_count_errors.cpp:40-136, fused into the
// decoders' write-out).
//
// Bit i of the data part is 1 when the codeword's posterior i is negative
// (neg(i)); word w of the hard decisions holds bits 32w..32w+31, LSB first.
// The warp builds word w with one ballot (lane = bit), lane w keeps it, and
// the error count is then word-level: lane w compares its word with the sent
// word w, and one warp reduction adds the bit errors.  A codeword error is
// counted per interleaved sub-codeword slot (i % z) % num_par
// (LDPC_count_errors.cpp:28-38,108-130): with num_par = 1 that is "any bit
// error"; otherwise lane w walks the error bits of its word.  Bits at or
// beyond kbits are 0 in both words.
#pragma once
#include <stdint.h>

namespace ldpc {

// hard_dst: the codeword's hard-decision words, or null; ref: its sent data
// words, or null (no counting).  Returns (in every lane) the bit errors in
// errw and the set of failing sub-codeword slots in errslots.
// PRELOAD: load the sent words of the first two rounds before the ballots
// (their latency then overlaps the ballots).  Measured: +3.8 % for the float
// decoder on 802.16e Z=96 (36 words, one codeword per CTA), -0.6 % for the
// int8 decoder on 802.11ad (11 words), which loads each round's words after
// its ballots.
template <bool PRELOAD, class NegF>
__device__ __forceinline__ void warp_hard_decisions(NegF neg, int kbits, int hard_words, int z, int num_par,
                                                    uint32_t* hard_dst, const uint32_t* ref, int lane,
                                                    unsigned& errw, unsigned& errslots) {
    errw = 0;
    errslots = 0;
    uint32_t sent_next = 0, sent_after = 0;
    if (PRELOAD) {
        sent_next = (ref && lane < hard_words) ? ref[lane] : 0u;
        sent_after = (ref && 32 + lane < hard_words) ? ref[32 + lane] : 0u;
    }
    for (int w0 = 0; w0 < hard_words; w0 += 32) {
        const int wn = min(32, hard_words - w0);
        const bool own = lane < wn;
        uint32_t sent = 0;
        if (PRELOAD) {
            sent = sent_next;
            sent_next = sent_after;
            sent_after = (ref && w0 + 64 + lane < hard_words) ? ref[w0 + 64 + lane] : 0u;
        }
        uint32_t mine = 0;
#pragma unroll 4
        for (int w = 0; w < wn; ++w) {
            const int i = (w0 + w) * 32 + lane;
            const uint32_t word = __ballot_sync(0xffffffffu, (i < kbits) && neg(i));
            if (lane == w) mine = word;
        }
        if (hard_dst && own) hard_dst[w0 + lane] = mine;
        if (ref) {
            if (!PRELOAD) sent = own ? ref[w0 + lane] : 0u;
            const int lo = (w0 + lane) * 32;
            uint32_t e = own ? (mine ^ sent) : 0u;
            if (own && lo + 32 > kbits) e &= (1u << (kbits - lo)) - 1u;
            errw += __reduce_add_sync(0xffffffffu, __popc(e));
            unsigned slots = 0;
            if (num_par == 1) {
                slots = e ? 1u : 0u;
            } else {
                for (uint32_t x = e; x; x &= x - 1) slots |= 1u << (((lo + __ffs(x) - 1) % z) % num_par);
            }
            errslots |= __reduce_or_sync(0xffffffffu, slots);
        }
    }
}

}  // namespace ldpc
