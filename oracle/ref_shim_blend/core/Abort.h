// Shim (ours) standing in for waLBerla's core/Abort.h and debug macros when the
// reference's IcosahedralShellMap and p1_div_k_grad_blending_q3 form are compiled alone:
// an abort throws, asserts are off.
#pragma once
#include <sstream>
#include <stdexcept>

#define WALBERLA_ABORT( msg )                                                                                          \
   do                                                                                                                  \
   {                                                                                                                   \
      std::ostringstream walberlaAbortStream_;                                                                        \
      walberlaAbortStream_ << msg;                                                                                     \
      throw std::runtime_error( walberlaAbortStream_.str() );                                                         \
   } while ( 0 )
#define WALBERLA_UNUSED( x ) (void) ( x )
#define WALBERLA_ASSERT( x ) ( (void) 0 )
#define WALBERLA_ASSERT_EQUAL( a, b ) ( (void) 0 )
#define WALBERLA_ASSERT_GREATER( a, b ) ( (void) 0 )
