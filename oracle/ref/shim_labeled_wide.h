/* Build shim: labeled reference with GRAPH_DEGREE raised so no candidate set
 * is truncated (the shipped value 4096 truncates, src/gpu_match.cu:302). */
#include <cstddef>
#define GRAPH_DEGREE GRAPH_DEGREE_AS_SHIPPED
#include "config.h"
#undef GRAPH_DEGREE
inline constexpr size_t GRAPH_DEGREE = 16384;
inline constexpr bool PACKAGE_ONLY = false;
