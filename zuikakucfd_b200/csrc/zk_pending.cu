// Entry points of drivers not built yet: they report ZK_ERR_UNSUPPORTED.
#include "zk_internal.h"

int zk_dg_setup(zk_ctx*) { return zk_internal_fail(ZK_ERR_UNSUPPORTED, "DG path not built yet"); }
void zk_dg_release(zk_ctx*) {}
int zk_dg_step(zk_ctx*, double) { return zk_internal_fail(ZK_ERR_UNSUPPORTED, "DG path not built yet"); }
int zk_dg_rhs(zk_ctx*, double*) { return zk_internal_fail(ZK_ERR_UNSUPPORTED, "DG path not built yet"); }
int zk_dg_limit(zk_ctx*) { return zk_internal_fail(ZK_ERR_UNSUPPORTED, "DG path not built yet"); }
