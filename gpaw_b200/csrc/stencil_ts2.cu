// stencil_ts2.cu -- star_tmasplit_kernel instantiations for 2 column group(s)
// of 32 (one translation unit per count, so they compile in parallel).
#include "stencil_tmasplit.cuh"

GFD_DEFINE_TS_ENTRY(2)
