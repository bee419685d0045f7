// Overlap collisions (placeholder until the collision kernels land).
#include "gtd_system.cuh"
using namespace gtd;
void release_collide(gtd_system *s) { cudaFree(s->coll_buf); s->coll_buf = nullptr; s->coll_bytes = 0; }
int run_collisions(gtd_system *) { return fail(GTD_ERR_UNSUPPORTED, "collisions not built"); }
