// stubs.cu -- entry points whose kernels are not built yet report
// FG_ERR_UNSUPPORTED (never a CPU fallback).
#include "runtime.h"

using namespace fgrt;
extern "C" {
}
