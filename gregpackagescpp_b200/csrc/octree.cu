// Barnes-Hut octree (placeholder until the linear-octree kernels land).
#include "gtd_system.cuh"
using namespace gtd;
void release_tree(gtd_system *s) { cudaFree(s->tree_buf); s->tree_buf = nullptr; s->tree_bytes = 0; s->tree_valid = false; }
int bh_evolve_kdk(gtd_system *, uint64_t) { return fail(GTD_ERR_UNSUPPORTED, "Barnes-Hut not built"); }
int bh_accelerations(gtd_system *, double *, uint32_t *) { return fail(GTD_ERR_UNSUPPORTED, "Barnes-Hut not built"); }
extern "C" {
int gtd_bh_build(gtd_system *, int) { return fail(GTD_ERR_UNSUPPORTED, "Barnes-Hut not built"); }
int gtd_bh_tree_size(gtd_system *, int64_t *, int64_t *, double *) { return fail(GTD_ERR_UNSUPPORTED, "Barnes-Hut not built"); }
int gtd_bh_tree_download(gtd_system *, uint64_t *, int32_t *, int8_t *, int8_t *, int32_t *, int32_t *, int32_t *, double *, double *, double *) { return fail(GTD_ERR_UNSUPPORTED, "Barnes-Hut not built"); }
int gtd_bh_accelerations(gtd_system *, double *, uint32_t *) { return fail(GTD_ERR_UNSUPPORTED, "Barnes-Hut not built"); }
}
