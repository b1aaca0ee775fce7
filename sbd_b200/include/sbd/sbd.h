/*
 * Drop-in umbrella header: a program written against the reference
 * (#include "sbd/sbd.h", r-ccs-cms/sbd include/sbd/sbd.h) builds against the
 * B200 path by putting sbd_b200/include and include/ on its include path and
 * linking sbd_b200/libsbdgpu.so.  It provides the tensor-product-basis entry
 * point sbd::tpb::diag and the input/output helpers around it, and the
 * generic second-quantised path (GeneralOp, Basis, mult, Lanczos).
 */
#ifndef SBD_GPU_UMBRELLA_SBD_H
#define SBD_GPU_UMBRELLA_SBD_H
#include "sbd_gpu/tpb.h"
#include "sbd_gpu/generalop.h"
#endif
