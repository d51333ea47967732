// Build-variant header for the FP64 grid oracle: identical declarations to
// the reference's include/shiokaze/core/config.h (same names and array cores)
// except that Real is double. Placed ahead of the reference include path.
#ifndef SHKZ_CONFIG_H
#define SHKZ_CONFIG_H
SHKZ_BEGIN_NAMESPACE
using Real = double;
const static char *shkz_default_array_core2 = "tiledarray2";
const static char *shkz_default_array_core3 = "tiledarray3";
SHKZ_END_NAMESPACE
#endif
