/* Test build of the drop-in dmrg_b200/dropin/dmrgx_znaupd.cpp against the
 * reference sources.  TEST INFRASTRUCTURE ONLY.
 *
 * A maintainer adds one friend declaration to the reference's include/qtensor.h
 * so that the drop-in can read a qtensor's blocks.  The reference tree is
 * read-only here, so this unit opens the class's private members while it
 * includes the reference headers instead, then compiles the drop-in file as
 * it is.  The oracle variants *_dropin link it with the unmodified reference
 * sources and libdmrgx.so in place of the ARPACK hook (oracle/Makefile).
 */
#include "global.h"
#include <algorithm>
#include <complex>
#include <iostream>
#include <vector>
#define private public
#include "qtensor.h"
#include "val_for_lanczos.h"
#undef private
#include "../dmrg_b200/dropin/dmrgx_znaupd.cpp"
