// NN-descent construction on the GPU (KGraphConstructor, kgraph.cpp:705-1001).
#include "kg_ctx.h"

using namespace kgb;

static unsigned g_verbosity = 1;

extern "C" {

void kg_set_verbosity(unsigned v) { g_verbosity = v; }

int kg_build(kg_ctx *ctx, const kg_index_params *params, kg_index_info *info) {
    (void)params; (void)info;
    return set_error(ctx, KG_E_RUNTIME, "build not available yet");
}

int kg_reverse(kg_ctx *ctx, int rev_k) {
    (void)rev_k;
    return set_error(ctx, KG_E_RUNTIME, "reverse not available yet");
}

int kg_prune(kg_ctx *ctx, unsigned level) {
    (void)level;
    return set_error(ctx, KG_E_RUNTIME, "prune not available yet");
}

}
