/* Build shim: the reference compiled with LABELED=false (its unlabeled mode),
 * without editing src/config.h.  The macro renames the shipped constant while
 * config.h is read (it is #pragma once, so later includes are skipped), then
 * the replacement value is declared.  Pre-included with -include. */
#include <cstddef>
#define LABELED LABELED_AS_SHIPPED
#include "config.h"
#undef LABELED
inline constexpr bool LABELED = false;
inline constexpr bool PACKAGE_ONLY = false;
