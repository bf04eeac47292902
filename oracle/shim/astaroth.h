/* Test infrastructure: stand-in for a DSL-generated or reference header; see ref_shim.h. */
#pragma once
#include "ref_shim.h"
