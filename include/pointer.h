/* pointer.h -- mirror of the reference header of the same name (olcf/minisweep
 * src/); the whole C API of the B200 sweep library is declared in
 * minisweep_b200.h, so the reference's own driver sources compile unchanged
 * against this directory. */
#ifndef MSB_MIRROR_POINTER_H
#define MSB_MIRROR_POINTER_H
#include "minisweep_b200.h"
#endif
