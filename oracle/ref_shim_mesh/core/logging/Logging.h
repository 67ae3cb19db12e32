// Shim (ours): see core/debug/CheckFunctions.h.
#pragma once
#include "core/debug/CheckFunctions.h"
