/* Single translation unit of the library: the __constant__ tables of
 * tg_aux.cu are visible to every kernel without relocatable device code. */
#include "tg_aux.cu"
#include "tg_tree.cu"
#include "tg_walk.cu"
#include "tg_gravity.cu"
#include "tg_adjoint.cu"
#include "tg_capi.cu"
#include "tg_batch.cu"
#include "tg_cosmo.cu"
#include "tg_load.cu"
#include "tg_fof.cu"
#include "tg_rung.cu"
#include "tg_noalloc.cu"
