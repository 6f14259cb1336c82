/* Build shim: labeled reference with GRAPH_DEGREE lowered to 16, so small
 * test graphs exercise its set truncation (src/gpu_match.cu:302,316). */
#include <cstddef>
#define GRAPH_DEGREE GRAPH_DEGREE_AS_SHIPPED
#include "config.h"
#undef GRAPH_DEGREE
inline constexpr size_t GRAPH_DEGREE = 16;
inline constexpr bool PACKAGE_ONLY = false;
