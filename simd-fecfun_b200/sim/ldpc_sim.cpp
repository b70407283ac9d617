// ldpc_sim -- process-level drop-in for the reference's LDPCtop_<variant>
// simulator (src/Top/LDPCtop.cpp:41-139), running on the GPU through
// libldpc_b200.so.  It speaks the same protocol, so build/run_LDPCsim.pl can
// drive it unchanged (exec=LDPCtop_Vec64c_min_b200, a link or copy of this
// binary):
//   stdin : the 820-byte sim_struct blob written by run_LDPCsim.pl:79-82 and
//           read by read_sim_params.cpp:12-27 (6 x 32-bit integers, 7 floats,
//           64 x 64-bit seeds, two 128-byte file names);
//   stdout: "CW Count: ..." (read_sim_params.cpp:32), "rand seed: ..." when it
//           draws its own seeds (:35-41), "Matrix Params: ..."
//           (encode_matrix_allocate.cpp:87), and after every outer loop one
//           "loop N: SNR=... inp_bit_err=... tot_iter=... tot_bit_err=...
//           tot_cw_err=... tot_dec_ticks=..." line per SNR point
//           (LDPCtop.cpp:127-129), which run_LDPCsim.pl:159-178 parses.
//
// The decoder variant comes from the program name, as the Perl driver reads
// it (run_LDPCsim.pl:51-66): Vec<n>c / s / w -> int8 / int16 / int32 offset
// min-sum, Vec<n>f / d -> float / double offset min-sum, or sum-product with
// "_prod".
//
// Differences from the reference, by design:
//   - noise and data come from Philox4x32-10 keyed by one 64-bit value that
//     is folded from the 64 seeds (splitmix64 over the seeds in order), so a
//     run with use_given_rand_state=1 and the printed seeds is repeatable;
//   - each outer loop decodes loop_count * num_codeword codewords per SNR
//     point in large GPU batches (the reference regenerates every inner
//     loop; the counts are the same sums);
//   - tot_dec_ticks is the decoder's device time converted to TSC ticks with
//     a TSC rate measured at start-up, so run_LDPCsim.pl's tick_freq
//     conversion still yields seconds;
//   - error counts print as 64-bit values;
//   - puncture_8023ca_flag is read and ignored, as in the reference
//     (gen_metrics.cpp:47 has it commented out).
#include <chrono>
#include <cinttypes>
#include <cstdio>
#include <cstdlib>
#include <cctype>
#include <cstring>
#include <random>
#include <string>
#include <thread>
#include <vector>
#include <x86intrin.h>

#include "ldpc_b200.h"

namespace {

#pragma pack(push, 1)
struct SimBlob {                   // read_sim_params.cpp:12-27, field by field
    uint32_t outer_count, loop_count, num_codeword, max_iter;
    int32_t puncture_8023ca_flag, use_given_rand_state;
    float max_row_metric, llr_scaling_factor, max_abs_llr, beta_offset, snr_start, snr_end, snr_step;
    uint64_t rand_state[64];
    char enc_raw_file[128];
    char dec_raw_file[128];
};
#pragma pack(pop)
static_assert(sizeof(SimBlob) == 820, "sim_struct blob is 820 bytes");

uint64_t splitmix64(uint64_t x) {
    x += 0x9e3779b97f4a7c15ull;
    x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ull;
    x = (x ^ (x >> 27)) * 0x94d049bb133111ebull;
    return x ^ (x >> 31);
}

uint64_t fold_seeds(const uint64_t* s) {
    uint64_t k = 0;
    for (int i = 0; i < 64; ++i) k = splitmix64(k ^ s[i]);
    return k;
}

double tsc_per_second() {
    const auto t0 = std::chrono::steady_clock::now();
    const unsigned long long c0 = __rdtsc();
    std::this_thread::sleep_for(std::chrono::milliseconds(50));
    const unsigned long long c1 = __rdtsc();
    const auto t1 = std::chrono::steady_clock::now();
    return (double)(c1 - c0) / std::chrono::duration<double>(t1 - t0).count();
}

[[noreturn]] void die(const char* what) {
    printf("ERROR: %s: %s\n", what, ldpc_last_error());
    fflush(stdout);
    exit(1);
}

// run_LDPCsim.pl:51-66 reads "Vec<lanes><type>" from the program name
// (c int8, s int16, w int32, f float, d double) and "_prod" for sum-product.
int variant_from_name(const char* argv0) {
    const std::string name = argv0 ? argv0 : "";
    const size_t v = name.rfind("Vec");
    char type = 'c';
    if (v != std::string::npos) {
        size_t i = v + 3;
        while (i < name.size() && isdigit((unsigned char)name[i])) ++i;
        if (i < name.size() && i > v + 3) type = name[i];
    }
    const bool prod = name.find("_prod") != std::string::npos;
    switch (type) {
        case 's': return LDPC_INT16_OMS;
        case 'w': return LDPC_INT32_OMS;
        case 'f': return prod ? LDPC_F32_SP : LDPC_F32_OMS;
        case 'd': return prod ? LDPC_F64_SP : LDPC_F64_OMS;
        default: return prod ? -1 : LDPC_INT8_OMS;
    }
}

}  // namespace

int main(int argc, char** argv) {
    (void)argc;
    SimBlob sim;
    if (fread(&sim, 1, sizeof(sim), stdin) != sizeof(sim)) {
        printf("Error in reading sim parameters from stdin!\n");
        return 1;
    }
    sim.enc_raw_file[127] = sim.dec_raw_file[127] = 0;
    printf("CW Count: %u codewords in inner loop * num_codeword\n", sim.loop_count * sim.num_codeword);
    if (sim.use_given_rand_state != 1) {
        std::random_device rd;
        for (int i = 0; i < 64; ++i) {
            sim.rand_state[i] = ((uint64_t)rd() << 32) ^ rd();
            printf("rand seed: %016" PRIx64 "\n", sim.rand_state[i]);
        }
    }
    const uint64_t seed = fold_seeds(sim.rand_state);

    ldpc_code* code = nullptr;
    if (ldpc_code_load_dat(sim.enc_raw_file, sim.dec_raw_file, &code) != LDPC_OK) die("loading the .dat tables");
    ldpc_code_info info;
    ldpc_code_get_info(code, &info);
    printf("Matrix Params: Z=%d  Hcol=%d  Hrow=%d num_par_cw=%d fill_cnt=%d\n", info.z, info.mcol, info.mrow,
           info.num_par, info.fill_cnt);
    fflush(stdout);

    ldpc_cfg cfg;
    cfg.variant = variant_from_name(argv[0]);
    if (cfg.variant < 0) {
        printf("ERROR: decoder variant of %s is not built (sum-product on integers)\n", argv[0]);
        return 1;
    }
    cfg.max_iter = sim.max_iter;
    cfg.max_row_metric = sim.max_row_metric;
    cfg.beta = sim.beta_offset;
    cfg.llr_scale = sim.llr_scaling_factor;
    cfg.max_abs_llr = sim.max_abs_llr;
    const char* dev_env = getenv("LDPC_DEVICE");
    ldpc_ctx* ctx = nullptr;
    if (ldpc_ctx_create(code, &cfg, dev_env ? atoi(dev_env) : 0, &ctx) != LDPC_OK) die("creating the decoder");

    // LDPCtop.cpp:75: SNR points SNR_start + k*SNR_step, k = 0..(end-start+1e-6)/step
    const unsigned last = sim.snr_step > 0 ? (unsigned)((sim.snr_end - sim.snr_start + 1e-6) / sim.snr_step) : 0;
    std::vector<float> snr(last + 1);
    for (unsigned k = 0; k <= last; ++k) snr[k] = k * sim.snr_step + sim.snr_start;
    if (snr.size() > 32) {
        printf("ERROR: %zu SNR points (at most 32)\n", snr.size());
        return 1;
    }
    const double tsc_hz = tsc_per_second();
    const unsigned long long per_outer = (unsigned long long)sim.loop_count * sim.num_codeword;
    std::vector<ldpc_snr_stats> st(snr.size());
    unsigned long long offset = 0;
    for (unsigned outloop = 0; outloop < sim.outer_count; ++outloop) {
        if (per_outer && ldpc_simulate(ctx, seed, offset, snr.data(), snr.size(), per_outer, st.data()) != LDPC_OK)
            die("simulating");
        if (!per_outer) memset(st.data(), 0, st.size() * sizeof(st[0]));
        offset += per_outer;
        for (size_t k = 0; k < snr.size(); ++k) {
            const long ticks = (long)(st[k].decode_ms * 1e-3 * tsc_hz);
            printf("loop %u: SNR=%f  inp_bit_err=%llu tot_iter=%llu tot_bit_err=%llu tot_cw_err=%llu tot_dec_ticks=%ld\n",
                   outloop, snr[k], st[k].uncoded_errors, st[k].iterations, st[k].bit_errors, st[k].cw_errors, ticks);
        }
        fflush(stdout);
    }
    ldpc_ctx_destroy(ctx);
    ldpc_code_destroy(code);
    return 0;
}
