// Empty stand-in: the vertex-DoF kernels include this header but use nothing from it.
#pragma once
