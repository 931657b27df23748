// batch_persist_d.cu -- the persistent decode kernel: the decode passes of batch_decode.cu compiled a
// second time with coherent loads (see batch_persist_c.cu).
#define GTSC_COHERENT_LOADS 1
#define GTSC_PERSISTENT_TU 1
#include "batch_decode.cu"
