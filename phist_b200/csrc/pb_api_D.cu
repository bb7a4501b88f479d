// pb_api_D.cu -- phist_D* entry points (double precision, _ST_ = _MT_ = double)
#include "pb_api.cuh"
#define PB_T double
#define PB_FN(name) phist_D##name
#define PB_XFN(name) phist_b200_D##name
#include "pb_api_inst.inc"
