// k_unet.cu -- learned warm start of the red-black projection.
#include "mdx_internal.cuh"

// ctx->guess holds the extrapolated increment; without a trained network it
// stays the guess.
int mdx_unet_guess(mdx_ctx_t* ctx, double dg, bool* made) {
    (void)ctx;
    (void)dg;
    (void)made;
    return MDX_OK;
}
