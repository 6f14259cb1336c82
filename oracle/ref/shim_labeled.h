/* Build shim for compiling the reference's own sources untouched.
 * The reference uses PACKAGE_ONLY (src/buffer.cu:266) without defining it;
 * this supplies the value its plot scripts assume (false).  Pre-included with
 * -include before any reference header. */
#include <cstddef>
#include "config.h"
inline constexpr bool PACKAGE_ONLY = false;
