"""A stand-in simulator process for the host-side driver tests: it reads the
820-byte blob and prints the reference's protocol lines (CW Count, Matrix
Params, one "loop" line per SNR point and outer loop) with counters that
depend only on the seeds, the outer loop and the SNR index, sleeping briefly
after every outer loop.  It never touches a GPU."""
import struct
import sys
import time

raw = sys.stdin.buffer.read(820)
if len(raw) != 820:
    print("Error in reading sim parameters from stdin!")
    sys.exit(1)
outer, inner, num_cw, max_iter, _, _ = struct.unpack_from("<6I", raw, 0)
_, _, _, _, s0, s1, step = struct.unpack_from("<7f", raw, 24)
seeds = struct.unpack_from("<64Q", raw, 52)
n_snr = int((s1 - s0 + 1e-6) / step) + 1 if step > 0 else 1
print("CW Count: %d codewords in inner loop * num_codeword" % (inner * num_cw), flush=True)
print("Matrix Params: Z=42  Hcol=16  Hrow=8 num_par_cw=1 fill_cnt=0", flush=True)
for o in range(outer):
    for k in range(n_snr):
        v = (seeds[0] + 7 * o + k) % 97
        print("loop %d: SNR=%f  inp_bit_err=%d tot_iter=%d tot_bit_err=%d tot_cw_err=%d tot_dec_ticks=%d"
              % (o, s0 + k * step, 1000 + v, 3 * inner * num_cw + v, v, v // 10, 12345), flush=True)
    time.sleep(0.05)
