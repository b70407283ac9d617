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
//
// Resume (no counterpart in the reference, whose driver appends each run's
// totals to ldpc_stat.m, run_LDPCsim.pl:140-153).  With LDPC_SIM_STATE=<file>
// the program rewrites <file> after every outer loop (a temporary file, then
// rename, so a kill leaves the previous state intact): a header with a hash
// of the run's parameters and the generator key, then every "loop N" line
// printed so far.  A later run with the same parameters (the outer count may
// differ) prints the saved lines first and continues at the next outer loop
// from the next codeword index; the generator is counter-based, so the
// counters equal those of an uninterrupted run.  A state of other
// parameters is reported and ignored.
#include <algorithm>
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
#include <unistd.h>
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

// FNV-1a over the parameters that fix a run's results: the blob without the
// outer count (and without the seeds when they are drawn afresh), plus the
// decoder variant.
uint64_t run_hash(SimBlob b, int variant) {
    b.outer_count = 0;
    if (b.use_given_rand_state != 1) memset(b.rand_state, 0, sizeof(b.rand_state));
    uint64_t h = 0xcbf29ce484222325ull;
    const unsigned char* p = reinterpret_cast<const unsigned char*>(&b);
    for (size_t i = 0; i < sizeof(b); ++i) h = (h ^ p[i]) * 0x100000001b3ull;
    return (h ^ (uint64_t)(uint32_t)variant) * 0x100000001b3ull;
}

struct SimState {
    uint64_t key = 0;                 // generator key of the saved run
    std::vector<std::string> lines;   // "loop N: ..." lines, n_snr per outer loop
};

// Reads a state file written for `hash`; false when absent or of another run.
bool read_state(const char* path, uint64_t hash, SimState* st) {
    FILE* f = fopen(path, "r");
    if (!f) return false;
    char buf[512];
    bool ok = false;
    unsigned long long h = 0, key = 0;
    if (fgets(buf, sizeof buf, f) && sscanf(buf, "ldpc_sim state v1 %llx %llx", &h, &key) == 2) {
        if (h == hash) {
            ok = true;
            st->key = key;
            while (fgets(buf, sizeof buf, f)) {
                std::string line(buf);
                while (!line.empty() && (line.back() == '\n' || line.back() == '\r')) line.pop_back();
                if (line.rfind("loop ", 0) == 0) st->lines.push_back(line);
            }
        } else {
            printf("state %s belongs to another run (parameters differ): ignored\n", path);
        }
    }
    fclose(f);
    return ok;
}

bool write_state(const char* path, uint64_t hash, const SimState& st) {
    const std::string tmp = std::string(path) + ".tmp";
    FILE* f = fopen(tmp.c_str(), "w");
    if (!f) return false;
    fprintf(f, "ldpc_sim state v1 %016" PRIx64 " %016" PRIx64 "\n", hash, st.key);
    for (const std::string& l : st.lines) fprintf(f, "%s\n", l.c_str());
    const bool ok = fflush(f) == 0 && fsync(fileno(f)) == 0;
    fclose(f);
    return ok && rename(tmp.c_str(), path) == 0;
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
    const int variant = variant_from_name(argv[0]);
    const char* state_path = getenv("LDPC_SIM_STATE");
    const uint64_t hash = run_hash(sim, variant);
    SimState state;
    const bool resumed = state_path && *state_path && read_state(state_path, hash, &state);
    uint64_t seed = state.key;
    if (!resumed) {
        if (sim.use_given_rand_state != 1) {
            std::random_device rd;
            for (int i = 0; i < 64; ++i) {
                sim.rand_state[i] = ((uint64_t)rd() << 32) ^ rd();
                printf("rand seed: %016" PRIx64 "\n", sim.rand_state[i]);
            }
        }
        seed = fold_seeds(sim.rand_state);
        state.key = seed;
    }

    ldpc_code* code = nullptr;
    if (ldpc_code_load_dat(sim.enc_raw_file, sim.dec_raw_file, &code) != LDPC_OK) die("loading the .dat tables");
    ldpc_code_info info;
    ldpc_code_get_info(code, &info);
    printf("Matrix Params: Z=%d  Hcol=%d  Hrow=%d num_par_cw=%d fill_cnt=%d\n", info.z, info.mcol, info.mrow,
           info.num_par, info.fill_cnt);
    fflush(stdout);
    if (variant < 0) {
        printf("ERROR: decoder variant of %s is not built (sum-product on integers)\n", argv[0]);
        return 1;
    }

    // LDPCtop.cpp:75: SNR points SNR_start + k*SNR_step, k = 0..(end-start+1e-6)/step
    const unsigned last = sim.snr_step > 0 ? (unsigned)((sim.snr_end - sim.snr_start + 1e-6) / sim.snr_step) : 0;
    std::vector<float> snr(last + 1);
    for (unsigned k = 0; k <= last; ++k) snr[k] = k * sim.snr_step + sim.snr_start;
    if (snr.size() > 32) {
        printf("ERROR: %zu SNR points (at most 32)\n", snr.size());
        return 1;
    }
    // outer loops already done by a saved run: print their lines again
    const unsigned done = std::min<unsigned>(sim.outer_count, (unsigned)(state.lines.size() / snr.size()));
    state.lines.resize((size_t)done * snr.size());
    for (const std::string& l : state.lines) printf("%s\n", l.c_str());
    fflush(stdout);
    if (done == sim.outer_count) {
        ldpc_code_destroy(code);
        return 0;
    }

    ldpc_cfg cfg;
    cfg.variant = variant;
    cfg.max_iter = sim.max_iter;
    cfg.max_row_metric = sim.max_row_metric;
    cfg.beta = sim.beta_offset;
    cfg.llr_scale = sim.llr_scaling_factor;
    cfg.max_abs_llr = sim.max_abs_llr;
    const char* dev_env = getenv("LDPC_DEVICE");
    ldpc_ctx* ctx = nullptr;
    if (ldpc_ctx_create(code, &cfg, dev_env ? atoi(dev_env) : 0, &ctx) != LDPC_OK) die("creating the decoder");

    const double tsc_hz = tsc_per_second();
    const unsigned long long per_outer = (unsigned long long)sim.loop_count * sim.num_codeword;
    std::vector<ldpc_snr_stats> st(snr.size());
    unsigned long long offset = (unsigned long long)done * per_outer;
    for (unsigned outloop = done; outloop < sim.outer_count; ++outloop) {
        if (per_outer && ldpc_simulate(ctx, seed, offset, snr.data(), snr.size(), per_outer, st.data()) != LDPC_OK)
            die("simulating");
        if (!per_outer) memset(st.data(), 0, st.size() * sizeof(st[0]));
        offset += per_outer;
        for (size_t k = 0; k < snr.size(); ++k) {
            const long ticks = (long)(st[k].decode_ms * 1e-3 * tsc_hz);
            char line[320];
            snprintf(line, sizeof line,
                     "loop %u: SNR=%f  inp_bit_err=%llu tot_iter=%llu tot_bit_err=%llu tot_cw_err=%llu tot_dec_ticks=%ld",
                     outloop, snr[k], st[k].uncoded_errors, st[k].iterations, st[k].bit_errors, st[k].cw_errors, ticks);
            printf("%s\n", line);
            state.lines.push_back(line);
        }
        fflush(stdout);
        if (state_path && *state_path && !write_state(state_path, hash, state))
            printf("warning: could not write the state file %s\n", state_path);
    }
    ldpc_ctx_destroy(ctx);
    ldpc_code_destroy(code);
    return 0;
}
