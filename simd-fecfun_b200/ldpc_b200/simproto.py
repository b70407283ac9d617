"""The reference simulator's process protocol, for driving ldpc_sim (or an
LDPCtop_* binary) from Python: the 820-byte stdin blob (run_LDPCsim.pl:79-82,
read by read_sim_params.cpp:12-27), the parse of the output lines
(run_LDPCsim.pl:159-178), and the generator key ldpc_sim folds from the 64
seeds."""
import re
import struct

LOOP_RE = re.compile(r"SNR=(\S+)\s+inp_bit_err=(\S+)\s+tot_iter=(\S+)\s+tot_bit_err=(\S+)\s+tot_cw_err=(\S+)\s+"
                     r"tot_dec_ticks=(\S+)")
MATRIX_RE = re.compile(r"Z=(\d+)  Hcol=(\d+)  Hrow=(\d+) num_par_cw=(\d+) fill_cnt=(\d+)")


def blob(outer, inner, num_cw, max_iter, mrm, scale, max_abs, beta, snr_start, snr_end, snr_step, seeds, enc, dec,
         given=1, punct8023=0):
    ints = struct.pack("<6I", outer, inner, num_cw, max_iter, punct8023, given)
    flts = struct.pack("<7f", mrm, scale, max_abs, beta, snr_start, snr_end, snr_step)
    name = lambda s: s.encode()[:127].ljust(128, b"\0")  # noqa: E731  (Perl pack 'Z128')
    return ints + flts + struct.pack("<64Q", *seeds) + name(enc) + name(dec)


def parse(text):
    out = {"loops": []}
    for line in text.splitlines():
        if line.startswith("CW Count"):
            out["cw_count"] = int(re.match(r"^CW Count: (\d+)", line).group(1))
        elif line.startswith("Matrix Params"):
            out["matrix"] = tuple(int(v) for v in MATRIX_RE.search(line).groups())
        elif line.startswith("loop"):
            v = LOOP_RE.search(line).groups()
            out["loops"].append((float(v[0]), int(v[1]), int(v[2]), int(v[3]), int(v[4]), int(v[5])))
    return out


def fold_seeds(seeds):
    """The 64-bit generator key ldpc_sim derives from the 64 seeds."""
    m = (1 << 64) - 1
    k = 0
    for s in seeds:
        x = (k ^ s) & m
        x = (x + 0x9E3779B97F4A7C15) & m
        x = ((x ^ (x >> 30)) * 0xBF58476D1CE4E5B9) & m
        x = ((x ^ (x >> 27)) * 0x94D049BB133111EB) & m
        k = x ^ (x >> 31)
    return k


def run_hash(blob_bytes: bytes, variant: int) -> int:
    """The parameter hash ldpc_sim writes in its state file header (FNV-1a
    over the blob with the outer count zeroed, and the seeds zeroed unless
    use_given_rand_state is 1, then the decoder variant)."""
    b = bytearray(blob_bytes)
    b[0:4] = b"\0\0\0\0"
    if struct.unpack_from("<i", b, 20)[0] != 1:
        b[52:52 + 512] = bytes(512)
    m = (1 << 64) - 1
    h = 0xCBF29CE484222325
    for v in b:
        h = ((h ^ v) * 0x100000001B3) & m
    return ((h ^ (variant & 0xFFFFFFFF)) * 0x100000001B3) & m


def state_text(blob_bytes: bytes, variant: int, key: int, lines) -> str:
    """A state file as ldpc_sim writes it (LDPC_SIM_STATE)."""
    return "ldpc_sim state v1 %016x %016x\n" % (run_hash(blob_bytes, variant), key) + "".join(l + "\n" for l in lines)
