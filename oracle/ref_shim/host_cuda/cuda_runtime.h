/* Host build of the reference kernels: everything CUDA-specific they use is
 * provided by ref_prelude_cpu.h (forced include).  Checker shim. */
#pragma once
