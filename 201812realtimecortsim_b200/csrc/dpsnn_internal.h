// dpsnn_internal.h -- declarations shared by the engine's translation units.
#pragma once
#include <stdint.h>
#include "../../include/dpsnn_b200.h"

// Record a message for dpsnn_last_error() and return `code`.
int dpsnn_fail(int code, const char *fmt, ...);

// Directory of the loaded library (for data files shipped beside it).
const char *dpsnn_library_dir(void);
