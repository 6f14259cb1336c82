/* Build shim: unlabeled reference with GRAPH_DEGREE lowered to 16. */
#include <cstddef>
#define LABELED LABELED_AS_SHIPPED
#define GRAPH_DEGREE GRAPH_DEGREE_AS_SHIPPED
#include "config.h"
#undef LABELED
#undef GRAPH_DEGREE
inline constexpr bool LABELED = false;
inline constexpr size_t GRAPH_DEGREE = 16;
inline constexpr bool PACKAGE_ONLY = false;
