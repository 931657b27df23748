// batch_persist_c.cu -- the persistent compress kernel (batch.hpp, PUnit): the compress passes of
// batch_kernels.cu compiled a second time with coherent loads.  In one persistent launch a pass
// reads what earlier passes of the same launch wrote, which the read-only (non-coherent) path the
// stage kernels use does not allow.
#define GTSC_COHERENT_LOADS 1
#define GTSC_PERSISTENT_TU 1
#include "batch_kernels.cu"
