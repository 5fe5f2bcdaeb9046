// inst.cu -- compiled once per K with -DCF_K=<K> (see build.py); instantiates that K's kernels.
#ifndef CF_K
#error "compile with -DCF_K=<K>"
#endif
#include "inst.cuh"
