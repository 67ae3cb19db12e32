// Shim (ours): see CheckFunctions.h.
#pragma once
#include "core/debug/CheckFunctions.h"
