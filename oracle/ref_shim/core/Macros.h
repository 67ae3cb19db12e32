// Minimal stand-in for the waLBerla core header that the reference's generated
// macro-cell kernels include. Only the restrict qualifier is needed.
#pragma once
#define WALBERLA_RESTRICT __restrict__
