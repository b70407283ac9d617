"""ldpc_decode_set_compat as a literal drop-in for LDPCdecode_set
(LDPCdecode.cpp:203-245) for every element type: the reference's own
pipeline (normdist2, gen_rand_databits, LDPCencode, gen_metrics; built from
its sources in oracle/_ref) fills its padded metrics buffer; one copy is
decoded in place by the reference, the other by the GPU through the compat
entry point with the build's lane count.  Sum of iterations and every
element of the Z-element column regions must agree."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

# build, Context variant name, element bits, (max_row_metric, beta, LLR scale, max|LLR|) as the Perl driver sets them
CASES = [
    ("Vec64c_min", "LDPC_INT8_OMS", 8, (31.0, 1.0, 2.0, 24.0)),
    ("Vec32s_min", "LDPC_INT16_OMS", 16, (31.0, 1.0, 2.0, 24.0)),
    ("Vec16w_min", "LDPC_INT32_OMS", 32, (31.0, 1.0, 2.0, 24.0)),
    ("Vec16f_prod", "LDPC_F32_SP", 32, (6e-8, 0.0, 1.0, 1e9)),
    ("Vec16f_min", "LDPC_F32_OMS", 32, (31.0, 1.0, 2.0, 24.0)),
    ("Vec8d_prod", "LDPC_F64_SP", 64, (1e-16, 0.0, 1.0, 1e9)),
    ("Vec8d_min", "LDPC_F64_OMS", 64, (31.0, 1.0, 2.0, 24.0)),
]


@pytest.mark.parametrize("build,variant,bits,params", CASES, ids=[c[0] for c in CASES])
@pytest.mark.parametrize("name,snr", [("11ad 1/2", -0.5), ("16e 1/2", 1.0)])
def test_compat_matches_reference_in_place(capi, build, variant, bits, params, name, snr):
    import refbind as rb
    from ldpc_b200 import codes
    if not rb.ref_available(build):
        pytest.skip("reference build %s absent" % build)
    mrm, beta, scale, max_abs = params
    lib = rb.RefLib(build)
    code = codes.make_code(name, elem_size=bits)
    n = 48
    ref = rb.RefCtx(lib, code, n)
    seeds = (np.arange(64, dtype=np.uint64) + np.uint64(77)) * np.uint64(0x9E3779B97F4A7C15) | np.uint64(1)
    rb.ref_init_randstate(lib, seeds)
    wgn = rb.ref_normdist2(lib, ref.wgn_count())
    ref.gen_rand_databits()
    ref.encode()
    ref.gen_metrics(snr, wgn, scale, max_abs)
    ours = ref.metrics.copy()
    tot_ref = ref.decode_set(10, mrm, beta)
    ctx = capi.Context(capi.Code.from_tables(code), variant=getattr(capi, variant), max_iter=10, max_row_metric=mrm,
                       beta=beta, llr_scale=scale, max_abs_llr=max_abs)
    tot = ctx.decode_set_compat(ours, n, lib.simd_par)
    P = lib.simd_par
    assert tot == tot_ref
    a = ref.metrics[:, :, P:P + code.z]
    b = ours[:, :, P:P + code.z]
    if a.dtype.kind == "f":
        assert np.array_equal(a.view(np.uint8), b.view(np.uint8))
    else:
        assert np.array_equal(a, b)
