// Shim (ours) standing in for waLBerla's check and debug macros when the reference's
// MeshGenSphericalShell.cpp is compiled alone: an abort throws, asserts are off.
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
#define WALBERLA_ASSERT_EQUAL( ... ) ( (void) 0 )
#define WALBERLA_ASSERT_LESS( ... ) ( (void) 0 )
#define WALBERLA_ASSERT_GREATER( ... ) ( (void) 0 )
#define WALBERLA_ASSERT_NULLPTR( ... ) ( (void) 0 )
#define WALBERLA_ASSERT_NOT_NULLPTR( ... ) ( (void) 0 )
