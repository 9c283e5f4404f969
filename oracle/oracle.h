/* Oracle: hand-written CPU restatement of the hot-path kernels (test infrastructure). */
#pragma once
#include <stdint.h>
#include <stddef.h>
uint32_t te_fnv1a(const uint32_t* w, size_t n);
