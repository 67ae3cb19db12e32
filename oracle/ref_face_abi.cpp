// Test infrastructure: a plain-pointer C ABI around the reference's own, unmodified
// generated macro-face kernels (compiled from the reference source tree by
// oracle/Makefile into oracle/_ref/). Only the golden-fixture generator uses it; it is
// never part of the product path.
//
// Kernels wrapped (paths relative to the reference project root):
//   src/hyteg/p1functionspace/generatedKernels/apply_3D_macroface_one_sided_vertexdof_to_vertexdof_{replace,add}.cpp
//   src/hyteg/p1functionspace/generatedKernels/sor_3D_macroface_P1{,_backwards}.cpp            (two-sided)
//   src/hyteg/p1functionspace/generatedKernels/sor_3D_macroface_P1_one_sided{,_backwards}.cpp  (one-sided)
//   src/hyteg/p1functionspace/generatedKernels/communicate_directly_vertexdof_{cell_to_face,face_to_cell}.cpp
//
// Face memory (P1ConstantOperator.cpp:208-306, VertexDoFPackInfo.hpp:540-600): the face's
// closure points as a triangle of width 2^L + 1 (row j, point i at
// i + j (2^L + 2) - j (j + 1) / 2), then one ghost layer per neighbour cell as a triangle of
// width 2^L (the cell's points at distance one from the face, in the face's coordinates).
// A neighbour cell is described by the cell-local ids of the face's vertices 0, 1, 2
// (Cell::getFaceLocalVertexToCellLocalVertexMaps), its stencil by 15 weights keyed by
// cell-logical offsets in the order
//   0:(0,0,0) 1:(1,0,0) 2:(-1,0,0) 3:(0,1,0) 4:(0,-1,0) 5:(0,0,1) 6:(0,0,-1)
//   7:(-1,1,0) 8:(1,-1,0) 9:(-1,0,1) 10:(1,0,-1) 11:(0,-1,1) 12:(0,1,-1)
//   13:(-1,1,-1) 14:(1,-1,1)
#include <cstdint>
#include <map>

#include "hyteg/p1functionspace/generatedKernels/apply_3D_macroface_one_sided_vertexdof_to_vertexdof_add.hpp"
#include "hyteg/p1functionspace/generatedKernels/apply_3D_macroface_one_sided_vertexdof_to_vertexdof_replace.hpp"
#include "hyteg/p1functionspace/generatedKernels/communicate_directly_vertexdof_cell_to_face.hpp"
#include "hyteg/p1functionspace/generatedKernels/communicate_directly_vertexdof_face_to_cell.hpp"
#include "hyteg/p1functionspace/generatedKernels/sor_3D_macroface_P1.hpp"
#include "hyteg/p1functionspace/generatedKernels/sor_3D_macroface_P1_backwards.hpp"
#include "hyteg/p1functionspace/generatedKernels/sor_3D_macroface_P1_one_sided.hpp"
#include "hyteg/p1functionspace/generatedKernels/sor_3D_macroface_P1_one_sided_backwards.hpp"

namespace {
const int kOffsets[15][3] = { { 0, 0, 0 },   { 1, 0, 0 },  { -1, 0, 0 }, { 0, 1, 0 },  { 0, -1, 0 },
                              { 0, 0, 1 },   { 0, 0, -1 }, { -1, 1, 0 }, { 1, -1, 0 }, { -1, 0, 1 },
                              { 1, 0, -1 },  { 0, -1, 1 }, { 0, 1, -1 }, { -1, 1, -1 }, { 1, -1, 1 } };

std::map< hyteg::indexing::Index, double > toMap( const double* st )
{
   std::map< hyteg::indexing::Index, double > m;
   for ( int o = 0; o < 15; ++o )
      m[hyteg::indexing::Index( kOffsets[o][0], kOffsets[o][1], kOffsets[o][2] )] = st[o];
   return m;
}

// (a0, a1, a2) > (b0, b1, b2) lexicographically
bool idsGreater( const int* a, const int* b )
{
   if ( a[0] != b[0] )
      return a[0] > b[0];
   if ( a[1] != b[1] )
      return a[1] > b[1];
   return a[2] > b[2];
}
} // namespace

extern "C" {

// One neighbour cell's share of the face apply (replace for the first cell, add for the
// second, as apply_face3D_generated does).
void ref_face_apply( double* dst, const double* src, const double* gl, int level, const int* ids, const double* st15,
                     int add )
{
   using namespace hyteg::vertexdof::macroface::generated;
   if ( add )
      apply_3D_macroface_one_sided_vertexdof_to_vertexdof_add( dst, src, gl, level, ids[0], ids[1], ids[2], toMap( st15 ) );
   else
      apply_3D_macroface_one_sided_vertexdof_to_vertexdof_replace(
          dst, src, gl, level, ids[0], ids[1], ids[2], toMap( st15 ) );
}

// Face SOR sweep as smooth_sor_face3D_generated (P1ConstantOperator.cpp:372-534) calls it:
// one-sided when gl1 is null; two-sided with the neighbour whose local ids compare
// lexicographically smaller passed first.
void ref_face_sor( double* face, double* gl0, double* gl1, const double* rhs, int level, const int* ids0, const int* ids1,
                   double relax, const double* st0, const double* st1, int backwards )
{
   using namespace hyteg::vertexdof::macroface::generated;
   if ( gl1 == nullptr )
   {
      if ( backwards )
         sor_3D_macroface_P1_one_sided_backwards( face, gl0, rhs, level, ids0[0], ids0[1], ids0[2], relax, toMap( st0 ) );
      else
         sor_3D_macroface_P1_one_sided( face, gl0, rhs, level, ids0[0], ids0[1], ids0[2], relax, toMap( st0 ) );
      return;
   }
   double*       ga = gl0;
   double*       gb = gl1;
   const int*    ia = ids0;
   const int*    ib = ids1;
   const double* sa = st0;
   const double* sb = st1;
   if ( idsGreater( ids0, ids1 ) )
   {
      ga = gl1;
      gb = gl0;
      ia = ids1;
      ib = ids0;
      sa = st1;
      sb = st0;
   }
   if ( backwards )
      sor_3D_macroface_P1_backwards(
          face, ga, gb, rhs, level, ia[0], ia[1], ia[2], ib[0], ib[1], ib[2], relax, toMap( sa ), toMap( sb ) );
   else
      sor_3D_macroface_P1( face, ga, gb, rhs, level, ia[0], ia[1], ia[2], ib[0], ib[1], ib[2], relax, toMap( sa ), toMap( sb ) );
}

// Ghost layer of one neighbour cell (VertexDoFPackInfo::communicateLocalCellToFace).
void ref_cell_to_face( const double* cell, double* gl, int level, const int* ids )
{
   hyteg::vertexdof::comm::generated::communicate_directly_vertexdof_cell_to_face( cell, gl, level, ids[0], ids[1], ids[2] );
}

// Face closure into the cell's closure (VertexDoFPackInfo::communicateLocalFaceToCell).
void ref_face_to_cell( double* cell, const double* face, int level, const int* ids )
{
   hyteg::vertexdof::comm::generated::communicate_directly_vertexdof_face_to_cell( cell, face, level, ids[0], ids[1], ids[2] );
}

} // extern "C"
