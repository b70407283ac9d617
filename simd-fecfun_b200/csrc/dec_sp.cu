// Host side of the float decoders (filled in with the sum-product kernel).
#include "internal.h"
namespace ldpc {
int setup_sp(ldpc_ctx* x) { (void)x; return fail(LDPC_ERR_UNSUPPORTED, "float decoders not built yet"); }
int launch_sp(ldpc_ctx* x, const DecodeArgs& a, cudaStream_t s) { (void)x; (void)a; (void)s; return fail(LDPC_ERR_UNSUPPORTED, "float decoders not built yet"); }
}  // namespace ldpc
