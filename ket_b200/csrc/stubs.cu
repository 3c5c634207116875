// stubs.cu -- entry points not yet implemented (return KET_ERR_UNSUPPORTED).
#include "ctx.h"

using namespace ket;

extern "C" {

}
