// Serving loop: continuous batching of independent multigrid solves on one GPU.
//
// No reference counterpart: the reference runs one GeometricMultigridSolver solve per MPI
// job (GeometricMultigridSolver.hpp:136-235 driven by an app's main loop). Here one host
// thread admits requests by device footprint, keeps their level hierarchies resident,
// and runs every admitted solve on the solve's own stream as ONE captured CUDA graph: a
// WHILE node around a V-cycle (FP64) or refinement step (mixed precision) and a device-side
// stopping test (runSolveLoop), so a solve costs the host one launch and one event. Small
// hierarchies (whole V-cycles in the one-block program kernel) are batched instead: the
// small requests admitted in one round of the loop run in ONE launch of k_solve_batch, a
// thread block per solve carrying it from its start residual to its tolerance, so a batch
// of small solves costs one launch in all. Whenever a solve finishes the loop admits newly
// arrived requests, and the GPU interleaves the kernels of all solves in flight.
//
// Included at the end of hyb_capi.cu (same translation unit: it uses the engine's
// internal types and launchers).

#include <chrono>
#include <deque>
#include <thread>

namespace hyb {

constexpr int    kServeModes   = 64;  // random Fourier features of the lognormal coefficient
constexpr double kServeCorrLen = 0.2; // correlation length of its Gaussian random field
constexpr double kServeSigma   = 1.0; // and its standard deviation
constexpr int    kServePre = 3, kServePost = 3;
constexpr double kServeCoarseTol     = 1e-12;
// hierarchies whose finest level holds at most this many closure points (all cells) run
// whole V-cycles in the program kernel
constexpr long   kServeProgramPoints = 65536;
constexpr int    kServeCoarseMaxIter = 10000;

inline uint64_t splitmix64Host( uint64_t x )
{
   x += 0x9E3779B97F4A7C15ull;
   uint64_t z = x;
   z          = ( z ^ ( z >> 30 ) ) * 0xBF58476D1CE4E5B9ull;
   z          = ( z ^ ( z >> 27 ) ) * 0x94D049BB133111EBull;
   return z ^ ( z >> 31 );
}

// w (modes x 3) ~ N(0, 1/corrLen^2) and phase ~ U[0, 2 pi): the i-th uniform of the stream is
// splitmix64( key + i ) scaled to (0, 1]; normals by the Box-Muller transform.
void rffFeatures( uint64_t seed, double corrLen, int modes, double* w, double* phase )
{
   const uint64_t key = splitmix64Host( seed ^ 0x5EEDF00DCAFEull );
   uint64_t       i   = 0;
   auto           u01 = [&]() { return ( double( splitmix64Host( key + i++ ) >> 11 ) + 1.0 ) / 9007199254740992.0; };
   const double   twoPi = 6.283185307179586476925286766559;
   for ( int m = 0; m < 3 * modes; ++m )
   {
      const double u1 = u01(), u2 = u01();
      w[m]            = std::sqrt( -2.0 * std::log( u1 ) ) * std::cos( twoPi * u2 ) / corrLen;
   }
   for ( int m = 0; m < modes; ++m )
      phase[m] = twoPi * ( u01() - 0.5 / 9007199254740992.0 );
}

struct ServeKey
{
   int  nx, ny, nz, level, coeff, precision, mesh;
   bool sameMesh( const ServeKey& o ) const { return mesh == o.mesh && nx == o.nx && ny == o.ny && nz == o.nz; }
   long cells() const
   {
      return mesh == HYB_MESH_SHELL ? 60l * ( nx - 1 ) * ( nx - 1 ) * ( ny - 1 ) : 6l * nx * ny * nz;
   }
   bool operator==( const ServeKey& o ) const
   {
      return sameMesh( o ) && level == o.level && coeff == o.coeff && precision == o.precision;
   }
};

inline long long gcdll( long long a, long long b ) { return b == 0 ? a : gcdll( b, a % b ); }

inline double serveLattice( const ServeKey& k )
{
   if ( k.mesh == HYB_MESH_SHELL )
      return double( 1 << 20 ); // shell points are not on a lattice: a fine one
   long long l = k.nx;
   l           = l / gcdll( l, k.ny ) * k.ny;
   l           = l / gcdll( l, k.nz ) * k.nz;
   return double( l << k.level );
}

// Device bytes of one resident hierarchy, an upper bound of what Instance allocates: per
// level the solution, right-hand side and GMG residual (FP64); for mixed precision the FP64
// refinement residual and the FP32 solution, right-hand side and residual; for the
// lognormal coefficient its FP64 and FP32 nodal values and the micro-tet matrices. Level 0
// adds the CG scratch (and the FP64 copies of the FP32 coarse problem); every solver has
// its own partial-sum array for dot products.
size_t serveFootprint( const ServeKey& k, int meshMaxLevel )
{
   const size_t nC  = size_t( k.cells() );
   size_t       per = 3 * 8;
   if ( k.precision == 32 )
      per += 8 + 3 * 4;
   if ( k.coeff != HYB_COEFF_CONSTANT )
      per += 8 + 4;
   size_t bytes = 0;
   for ( int l = 0; l <= k.level; ++l )
   {
      const size_t N = size_t( 1 ) << l;
      const size_t S = ( N + 1 ) * ( N + 2 ) * ( N + 3 ) / 6;
      bytes += nC * size_t( stridePad( int( S ) ) ) * per;
      if ( k.coeff != HYB_COEFF_CONSTANT )
         bytes += nC * 96 * ( 8 + 4 );
   }
   bytes += nC * size_t( stridePad( 4 ) ) * 8 * ( k.precision == 32 ? 5 : 3 );
   size_t maxPartial = 1;
   for ( int l = 0; l <= meshMaxLevel; ++l )
   {
      const size_t N = size_t( 1 ) << l;
      const size_t S = ( N + 1 ) * ( N + 2 ) * ( N + 3 ) / 6;
      maxPartial     = std::max( maxPartial, ( S + 255 ) / 256 * nC );
   }
   bytes += maxPartial * 8 + 2 * 8 + 4 * sizeof( int ) + 4 * kServeModes * 8;
   // an allowance of 64 KiB per level for the recorded phase list of the coarse-level
   // program kernel
   bytes += size_t( k.level + 1 ) * 65536;
   return bytes;
}

struct MeshEntry
{
   int                         nx, ny, nz, kind;
   std::unique_ptr< Storage >  st;
   std::unique_ptr< Operator > laplace;
   size_t                      bytes = 0;
};

// One resident hierarchy: everything a solve of one shape needs, reused by later requests
// of the same shape. The graphs its solver captured stay valid because every buffer keeps
// its address; a new request only rewrites the right-hand side and the coefficient.
struct Instance
{
   ServeKey                    key{};
   MeshEntry*                  mesh = nullptr;
   Operator*                   op   = nullptr;
   std::unique_ptr< Operator > ownOp; // lognormal coefficient
   std::unique_ptr< Gmg >      gmg;
   std::unique_ptr< Function > x, b;
   DevBuf< double >            feat;             // w (modes x 3) then phase (modes)
   double*                     featHost = nullptr; // pinned
   cudaStream_t                stream   = nullptr;
   cudaEvent_t                 ev       = nullptr;
   size_t                      bytes    = 0;
   uint64_t                    lastUse  = 0;
   int                         req      = -1; // request being served, -1 when idle
   bool                        hostLoop = false; // the device-iterated solve graph is unavailable
   bool                        batch    = false; // solved in k_solve_batch with the small solves admitted beside it
   const Gmg::Program*         solveProg = nullptr; // its whole-solve program (batch)

   ~Instance()
   {
      if ( stream )
         cudaStreamSynchronize( stream );
      gmg.reset(); // its graphs reference the buffers below
      if ( ev )
         cudaEventDestroy( ev );
      if ( stream )
         cudaStreamDestroy( stream );
      if ( featHost )
         cudaFreeHost( featHost );
   }
};

enum ServeState : int
{
   kWaiting  = 0, // submitted, not yet arrived in a run
   kQueued   = 1, // arrived, waiting for a slot and memory
   kStarting = 2, // right-hand side, coefficient and initial residual enqueued
   kStepping = 3, // cycles in flight
   kDraining = 4, // solution copy to the host in flight
   kDone     = 5,
   kLooping  = 6  // the device-iterated solve and its result copy in flight
};

struct ServeRequest
{
   hyb_request d{};
   ServeKey    key{};
   double      arrival  = 0;
   double*     solution = nullptr;
   int         state    = kWaiting;
   int         status   = HYB_OK;
   int         cycles   = 0;
   double      nb = 1, rel = 0;
   double      tAdmit = 0, tDone = 0;
   size_t      footprint = 0, served = 0;
   Instance*   inst      = nullptr;
};

bool serveBatch();
bool serveHostLoop();

struct Server
{
   size_t                                    budget    = 0;
   int                                       maxActive = 1, maxLevel = 0;
   size_t                                    used = 0, peak = 0;
   int                                       built = 0, graphsEvicted = 0;
   int                                       batches = 0, batchedSolves = 0; // k_solve_batch launches, solves in them
   std::vector< cudaStream_t >               batchStreams; // batches of small solves, round robin
   int                                       batchNext = 0;

   ~Server()
   {
      for ( cudaStream_t b : batchStreams )
      {
         cudaStreamSynchronize( b );
         cudaStreamDestroy( b );
      }
   }

   cudaStream_t nextBatchStream()
   {
      constexpr int kBatchStreams = 8;
      if ( batchStreams.empty() )
         for ( int i = 0; i < kBatchStreams; ++i )
         {
            cudaStream_t b;
            HYB_CUDA( cudaStreamCreateWithFlags( &b, cudaStreamNonBlocking ) );
            batchStreams.push_back( b );
         }
      return batchStreams[size_t( batchNext++ % kBatchStreams )];
   }
   uint64_t                                  tick  = 0;
   std::vector< std::unique_ptr< MeshEntry > > meshes;
   std::vector< std::unique_ptr< Instance > >  inst;
   std::vector< ServeRequest >               reqs;

   void account( long long delta )
   {
      used = size_t( (long long) used + delta );
      peak = std::max( peak, used );
   }

   MeshEntry& mesh( const ServeKey& k )
   {
      for ( auto& m : meshes )
         if ( m->kind == k.mesh && m->nx == k.nx && m->ny == k.ny && m->nz == k.nz )
            return *m;
      const long long before = g_deviceBytes.load();
      auto            m      = std::make_unique< MeshEntry >();
      m->nx                  = k.nx;
      m->ny                  = k.ny;
      m->nz                  = k.nz;
      m->kind                = k.mesh;
      std::vector< std::array< double, 3 > > V;
      std::vector< std::array< int, 4 > >    T;
      const double                           lo[3] = { 0, 0, 0 }, hi[3] = { 1, 1, 1 };
      if ( k.mesh == HYB_MESH_SHELL )
         meshSphericalShell( k.nx, k.ny, 0.55, 1.0, V, T );
      else
         meshCuboid( k.nx, k.ny, k.nz, lo, hi, V, T );
      m->st = std::make_unique< Storage >();
      buildStorage( *m->st, V, T, maxLevel );
      m->laplace.reset( makeLaplace( m->st.get(), 0, maxLevel ) );
      // the mesh's row tables (shared by every hierarchy on it) belong to the mesh's bytes
      for ( int l = 0; l <= maxLevel; ++l )
         ensureRows( *m->st, l );
      m->bytes = size_t( g_deviceBytes.load() - before );
      account( (long long) m->bytes );
      meshes.push_back( std::move( m ) );
      return *meshes.back();
   }

   void evict( Instance* victim )
   {
      graphsEvicted += int( victim->gmg ? victim->gmg->graphs.size() + victim->gmg->loops.size() : 0 );
      const long long before = g_deviceBytes.load();
      for ( auto it = inst.begin(); it != inst.end(); ++it )
         if ( it->get() == victim )
         {
            inst.erase( it );
            break;
         }
      account( g_deviceBytes.load() - before );
   }

   Instance* build( const ServeKey& k )
   {
      MeshEntry&      me     = mesh( k );
      const long long before = g_deviceBytes.load();
      auto            in     = std::make_unique< Instance >();
      in->key                = k;
      in->mesh               = &me;
      Storage* st            = me.st.get();
      if ( k.coeff != HYB_COEFF_CONSTANT )
      {
         in->ownOp.reset( makeDivKGradWith( st, 0, k.level, []( int, double* ) {} ) );
         in->op = in->ownOp.get();
      }
      else
         in->op = me.laplace.get();
      in->gmg = std::make_unique< Gmg >();
      initGmg( *in->gmg, st, in->op, 0, k.level, kServePre, kServePost, 1.0, HYB_SMOOTHER_SOR, kServeCoarseTol,
               kServeCoarseMaxIter );
      // a small hierarchy runs every level of its V-cycle in the one-block program kernel:
      // its cost is launch latency, not bandwidth, and concurrent small solves then occupy
      // one multiprocessor each
      if ( long( st->td.nC ) * st->L( k.level ).dev.stride <= kServeProgramPoints )
         in->gmg->progTop = k.level;
      if ( k.precision == 32 )
         ensureMixed( *in->gmg );
      prepare( *in->gmg );
      in->x.reset( makeFunction( st, 0, k.level, HYB_F64 ) );
      in->b.reset( makeFunction( st, 0, k.level, HYB_F64 ) );
      // record the coarse-level program now, so that the hierarchy's footprint includes it
      Gmg& g = *in->gmg;
      if ( g.progTop >= 0 )
      {
         const int top = std::min( k.level, g.progTop );
         if ( k.precision == 32 )
            ensureProgram< float >( g, *g.x32, *g.b32, *g.t32, top );
         else
            ensureProgram< double >( g, *in->x, *in->b, *g.tmp64, top );
      }
      // a hierarchy whose whole V-cycle runs in the program kernel is solved by k_solve_batch
      // together with the other small solves admitted at the same time
      if ( g.progTop >= k.level && serveBatch() && !serveHostLoop() )
      {
         in->solveProg = ensureSolveProgram( g, *in->x, *in->b, k.level, k.precision == 64 ? kCycle64Norm : kMixedStep );
         in->batch     = true;
      }
      in->feat.alloc( 4 * kServeModes );
      HYB_CUDA( cudaMallocHost( &in->featHost, 4 * kServeModes * sizeof( double ) ) );
      HYB_CUDA( cudaStreamCreateWithFlags( &in->stream, cudaStreamNonBlocking ) );
      HYB_CUDA( cudaEventCreateWithFlags( &in->ev, cudaEventDisableTiming ) );
      HYB_CUDA( cudaDeviceSynchronize() );
      in->bytes = size_t( g_deviceBytes.load() - before );
      account( (long long) in->bytes );
      ++built;
      inst.push_back( std::move( in ) );
      return inst.back().get();
   }

   // An idle hierarchy of the request's shape, or a new one if its footprint fits the budget
   // once idle hierarchies are evicted least recently used first. nullptr: wait for running
   // solves to finish (or, with none running, the request can never fit).
   Instance* acquire( ServeRequest& r )
   {
      for ( auto& in : inst )
         if ( in->req < 0 && in->key == r.key )
            return in.get();
      mesh( r.key );
      while ( used + r.footprint > budget )
      {
         Instance* victim = nullptr;
         for ( auto& in : inst )
            if ( in->req < 0 && ( !victim || in->lastUse < victim->lastUse ) )
               victim = in.get();
         if ( !victim )
            break;
         evict( victim );
      }
      if ( used + r.footprint > budget )
         return nullptr;
      return build( r.key );
   }

   int graphsCaptured() const
   {
      int n = graphsEvicted;
      for ( auto& in : inst )
         n += int( in->gmg->graphs.size() + in->gmg->loops.size() );
      return n;
   }
};

void validateRequest( const Server& sv, const hyb_request& d )
{
   require( d.mesh == HYB_MESH_CUBOID || d.mesh == HYB_MESH_SHELL, "unknown mesh kind" );
   if ( d.mesh == HYB_MESH_CUBOID )
      require( d.nx >= 1 && d.ny >= 1 && d.nz >= 1 && d.nx <= 64 && d.ny <= 64 && d.nz <= 64,
               "macro-cubes per direction must be in [1, 64]" );
   else
      require( d.nx >= 2 && d.ny >= 2 && d.nx <= 64 && d.ny <= 64, "shell ntan and nrad must be in [2, 64]" );
   require( d.level >= 1 && d.level <= sv.maxLevel, "level must be in [1, the server's max_level]" );
   require( d.coefficient == HYB_COEFF_CONSTANT || d.coefficient == HYB_COEFF_LOGNORMAL ||
                d.coefficient == HYB_COEFF_RADIAL,
            "unknown coefficient kind" );
   require( d.precision == 64 || d.precision == 32, "precision must be 64 or 32" );
   require( d.rel_tol > 0 && std::isfinite( d.rel_tol ), "rel_tol must be positive" );
   require( d.max_cycles >= 1, "max_cycles must be at least 1" );
}

ServeKey keyOf( const hyb_request& d )
{
   const bool shell = d.mesh == HYB_MESH_SHELL;
   return ServeKey{ d.nx, d.ny, shell ? 1 : d.nz, d.level, d.coefficient, d.precision, d.mesh };
}

bool serveHostLoop();

// the request's right-hand side, coefficient and x = 0, on stream s
void setupRequest( Server& sv, ServeRequest& r, Instance& in, cudaStream_t s )
{
   const int L = r.key.level;
   Storage&  st = *in.mesh->st;
   in.req       = int( &r - sv.reqs.data() );
   in.lastUse   = ++sv.tick;
   r.inst       = &in;
   r.served     = in.bytes;
   if ( r.key.coeff != HYB_COEFF_CONSTANT )
   {
      const bool radial = r.key.coeff == HYB_COEFF_RADIAL;
      rffFeatures( r.d.seed, kServeCorrLen, kServeModes, in.featHost, in.featHost + 3 * kServeModes );
      HYB_CUDA( cudaMemcpyAsync( in.feat.p, in.featHost, 4 * kServeModes * sizeof( double ), cudaMemcpyHostToDevice, s ) );
      fillRff( *in.ownOp, in.feat.p, in.feat.p + 3 * kServeModes, kServeModes, radial ? 0.5 : kServeSigma,
               radial ? 5.0 : 0.0, s );
   }
   const auto& Lh = st.L( L );
   k_fill_uniform_hash< double ><<< dim3( Lh.slabBlocks, st.td.nC ), 256, 0, s >>>(
       st.td, Lh.dev, st.cellCoords.p, st.cellOrder.p, in.b->ptr< double >( L ), r.d.seed, serveLattice( r.key ) );
   HYB_CHECK_LAUNCH();
   HYB_CUDA( cudaMemsetAsync( in.x->ptr< double >( L ), 0, in.x->levelBytes( L ), s ) );
}

// set-up, ||b||^2, the initial residual norm, and (unless the hierarchy is stepped from the
// host) the whole solve as one device-iterated graph
void startRequest( Server& sv, ServeRequest& r, Instance& in )
{
   const int    L = r.key.level;
   cudaStream_t s = in.stream;
   Storage&     st = *in.mesh->st;
   setupRequest( sv, r, in, s );
   Gmg& g = *in.gmg;
   launchDot< double >( st, L, in.b->ptr< double >( L ), in.b->ptr< double >( L ), kGmgFlag, g.partial.p, g.scalars.p + 1,
                        s );
   runGraph( g, *in.x, *in.b, L, r.key.precision == 64 ? kNorm64 : kNormMixed, s );
   if ( !in.hostLoop && !serveHostLoop() )
   {
      // the whole solve as one graph launch with the stopping test on the device
      try
      {
         runSolveLoop( g, *in.x, *in.b, L, r.key.precision == 64 ? kCycle64Norm : kMixedStep, r.d.rel_tol,
                       r.d.max_cycles, s );
         HYB_CUDA( cudaMemcpyAsync( g.hostCtl, g.ctl.p, sizeof( SolveCtl ), cudaMemcpyDeviceToHost, s ) );
         HYB_CUDA( cudaEventRecord( in.ev, s ) );
         r.state = kLooping;
         return;
      }
      catch ( const Error& )
      {
         // the device loop could not be captured here: step this hierarchy from the host
         in.hostLoop = true;
         HYB_CUDA( cudaGetLastError() );
      }
   }
   HYB_CUDA( cudaMemcpyAsync( g.hostScalar, g.scalars.p, 2 * sizeof( double ), cudaMemcpyDeviceToHost, s ) );
   HYB_CUDA( cudaEventRecord( in.ev, s ) );
   r.state = kStarting;
}

// Start the small solves admitted together: their set-up and ONE k_solve_batch launch (per
// operator kind) on a stream of the batch pool, which runs each solve to its tolerance in
// its own thread block; then every solve's stopping-test state back to the host.
void startBatch( Server& sv, const std::vector< int >& ids )
{
   cudaStream_t            s = sv.nextBatchStream();
   std::vector< SolveJob > jobs[2];
   for ( int id : ids )
   {
      ServeRequest& r  = sv.reqs[size_t( id )];
      Instance&     in = *r.inst;
      setupRequest( sv, r, in, s );
      Gmg& g               = *in.gmg;
      g.hostCtl->tol       = r.d.rel_tol;
      g.hostCtl->maxCycles = r.d.max_cycles;
      HYB_CUDA( cudaMemcpyAsync( g.ctl.p, g.hostCtl, sizeof( SolveCtl ), cudaMemcpyHostToDevice, s ) );
      jobs[in.op->variable ? 1 : 0].push_back( solveJob( g, *in.solveProg ) );
   }
   for ( int v = 0; v < 2; ++v )
      if ( !jobs[v].empty() )
      {
         launchSolveBatch( jobs[v], v == 1, s );
         sv.batches += int( ( jobs[v].size() + kSolveBatchMax - 1 ) / kSolveBatchMax );
      }
   for ( int id : ids )
   {
      ServeRequest& r  = sv.reqs[size_t( id )];
      Instance&     in = *r.inst;
      HYB_CUDA( cudaMemcpyAsync( in.gmg->hostCtl, in.gmg->ctl.p, sizeof( SolveCtl ), cudaMemcpyDeviceToHost, s ) );
      HYB_CUDA( cudaEventRecord( in.ev, s ) );
      r.state = kLooping;
   }
   sv.batchedSolves += int( ids.size() );
}

// HYB_SERVE_BATCH=0: solve small hierarchies one device-iterated graph each instead of in
// k_solve_batch
bool serveBatch()
{
   static const bool v = envLong( "HYB_SERVE_BATCH", 1 ) != 0;
   return v;
}

// HYB_SERVE_HOST_LOOP=1: step every solve from the host (one graph launch and one residual
// read per cycle) instead of the device-iterated solve graph
bool serveHostLoop()
{
   static const bool v = envLong( "HYB_SERVE_HOST_LOOP", 0 ) != 0;
   return v;
}

// The request's last enqueued work has finished: take the device loop's result (or, stepped
// from the host, read the residual norm and enqueue the next step), then the solution copy,
// or finish. Returns true when the request is done.
bool advanceRequest( ServeRequest& r, double now )
{
   Instance& in = *r.inst;
   Gmg&      g  = *in.gmg;
   const int L  = r.key.level;
   if ( r.state == kDraining )
   {
      r.state = kDone;
      r.tDone = now;
      return true;
   }
   bool stop = false;
   if ( r.state == kLooping )
   {
      r.nb     = g.hostCtl->nb;
      r.rel    = g.hostCtl->rel;
      r.cycles = g.hostCtl->cycles;
      if ( !std::isfinite( r.rel ) || r.rel > r.d.rel_tol )
         r.status = HYB_ENOTCONVERGED;
      stop = true;
   }
   else
   {
      // stepped from the host: one cycle per event
      if ( r.state == kStarting )
      {
         r.nb    = std::sqrt( g.hostScalar[1] ) > 0 ? std::sqrt( g.hostScalar[1] ) : 1.0;
         r.state = kStepping;
      }
      r.rel = std::sqrt( g.hostScalar[0] ) / r.nb;
      if ( !std::isfinite( r.rel ) )
      {
         r.status = HYB_ENOTCONVERGED;
         stop     = true;
      }
      else if ( r.rel <= r.d.rel_tol )
         stop = true;
      else if ( r.cycles >= r.d.max_cycles )
      {
         r.status = HYB_ENOTCONVERGED;
         stop     = true;
      }
   }
   if ( !stop )
   {
      runGraph( g, *in.x, *in.b, L, r.key.precision == 64 ? kCycle64Norm : kMixedStep, in.stream );
      HYB_CUDA( cudaMemcpyAsync( g.hostScalar, g.scalars.p, sizeof( double ), cudaMemcpyDeviceToHost, in.stream ) );
      HYB_CUDA( cudaEventRecord( in.ev, in.stream ) );
      ++r.cycles;
      return false;
   }
   if ( r.solution )
   {
      // canonical DoF order staged in the solver's FP64 scratch, which the solve no longer needs
      Storage&     st = *in.mesh->st;
      const size_t n  = size_t( st.topo.numDofs( L ) );
      launchToDofs< double >( st, L, in.x->ptr< double >( L ), g.tmp64->ptr< double >( L ), in.stream );
      HYB_CUDA( cudaMemcpyAsync( r.solution, g.tmp64->ptr< double >( L ), n * sizeof( double ), cudaMemcpyDeviceToHost,
                                 in.stream ) );
      HYB_CUDA( cudaEventRecord( in.ev, in.stream ) );
      r.state = kDraining;
      return false;
   }
   r.state = kDone;
   r.tDone = now;
   return true;
}

void runServer( Server& sv, double timeLimit )
{
   using clk = std::chrono::steady_clock;
   std::vector< int > order;
   for ( size_t i = 0; i < sv.reqs.size(); ++i )
      if ( sv.reqs[i].state == kWaiting )
         order.push_back( int( i ) );
   std::stable_sort( order.begin(), order.end(),
                     [&]( int a, int b ) { return sv.reqs[a].arrival < sv.reqs[b].arrival; } );
   const auto t0      = clk::now();
   auto       elapsed = [&]() { return std::chrono::duration< double >( clk::now() - t0 ).count(); };
   size_t             next = 0;
   std::deque< int >  queue;
   std::vector< int > running;
   auto               release = [&]( ServeRequest& r ) {
      if ( r.inst )
      {
         r.inst->req     = -1;
         r.inst->lastUse = ++sv.tick;
      }
      r.inst = nullptr;
   };
   for ( ;; )
   {
      double now = elapsed();
      while ( next < order.size() && sv.reqs[order[next]].arrival <= now )
      {
         sv.reqs[order[next]].state = kQueued;
         queue.push_back( order[next++] );
      }
      // admission in arrival order, as slots and memory allow; small solves admitted in
      // the same round start as one batch
      std::vector< int > batch;
      while ( !queue.empty() && int( running.size() ) < sv.maxActive )
      {
         ServeRequest& r  = sv.reqs[queue.front()];
         Instance*     in = sv.acquire( r );
         if ( !in )
         {
            if ( !running.empty() )
               break;
            // nothing left to wait for: it cannot fit beside the resident meshes
            r.status = HYB_ENOMEM;
            r.state  = kDone;
            r.tAdmit = r.tDone = elapsed();
            queue.pop_front();
            continue;
         }
         queue.pop_front();
         r.tAdmit = elapsed();
         const int id = int( &r - sv.reqs.data() );
         if ( in->batch )
         {
            r.inst = in;
            in->req = id; // taken: a later request of the round must not acquire it
            batch.push_back( id );
         }
         else
            startRequest( sv, r, *in );
         running.push_back( id );
      }
      if ( !batch.empty() )
         startBatch( sv, batch );
      bool progressed = false;
      for ( size_t i = 0; i < running.size(); )
      {
         ServeRequest&     r = sv.reqs[running[i]];
         const cudaError_t q = cudaEventQuery( r.inst->ev );
         if ( q == cudaErrorNotReady )
         {
            ++i;
            continue;
         }
         HYB_CUDA( q );
         progressed = true;
         if ( advanceRequest( r, elapsed() ) )
         {
            release( r );
            running.erase( running.begin() + long( i ) );
         }
         else
            ++i;
      }
      if ( next == order.size() && queue.empty() && running.empty() )
         break;
      if ( elapsed() > timeLimit )
      {
         HYB_CUDA( cudaDeviceSynchronize() );
         for ( int id : order )
         {
            ServeRequest& r = sv.reqs[id];
            if ( r.state != kDone )
            {
               r.status = HYB_ETIMEOUT;
               r.state  = kDone;
               r.tDone  = elapsed();
               release( r );
            }
         }
         break;
      }
      if ( !progressed )
      {
         if ( running.empty() && queue.empty() && next < order.size() )
         {
            // idle until the next arrival
            const double wait = sv.reqs[order[next]].arrival - elapsed();
            if ( wait > 2e-4 )
               std::this_thread::sleep_for( std::chrono::duration< double >( wait - 1e-4 ) );
         }
         else
            std::this_thread::yield();
      }
   }
}

} // namespace hyb

struct hyb_server_s : hyb::Server
{};

extern "C" {

int hyb_server_create( size_t budget, int maxActive, int maxLevel, hyb_server** out )
{
   HYB_API_BEGIN
   require( out, "null argument" );
   require( budget > 0, "budget must be positive" );
   require( maxActive >= 1 && maxActive <= 1024, "max_active must be in [1, 1024]" );
   require( maxLevel >= 1 && maxLevel <= 9, "max_level must be in [1, 9]" );
   auto s       = std::make_unique< hyb_server_s >();
   s->budget    = budget;
   s->maxActive = maxActive;
   s->maxLevel  = maxLevel;
   *out         = s.release();
   HYB_API_END
}

int hyb_server_destroy( hyb_server* s )
{
   HYB_API_BEGIN
   if ( s )
   {
      if ( !s->inst.empty() )
         HYB_CUDA( cudaDeviceSynchronize() );
      delete static_cast< hyb_server_s* >( s );
   }
   HYB_API_END
}

int hyb_server_footprint( const hyb_server* s, const hyb_request* r, size_t* bytes )
{
   HYB_API_BEGIN
   require( s && r && bytes, "null argument" );
   validateRequest( *s, *r );
   *bytes = serveFootprint( keyOf( *r ), s->maxLevel );
   HYB_API_END
}

int hyb_server_submit( hyb_server* s, const hyb_request* r, double arrival, double* solution, int* id )
{
   HYB_API_BEGIN
   require( s && r, "null argument" );
   validateRequest( *s, *r );
   require( arrival >= 0 && std::isfinite( arrival ), "arrival time must be non-negative" );
   ServeRequest q;
   q.d         = *r;
   q.key       = keyOf( *r );
   q.arrival   = arrival;
   q.solution  = solution;
   q.footprint = serveFootprint( q.key, s->maxLevel );
   if ( q.footprint > s->budget )
      throw Error( HYB_ENOMEM, "request needs " + std::to_string( q.footprint ) + " device bytes, more than the budget of " +
                                   std::to_string( s->budget ) );
   s->reqs.push_back( q );
   if ( id )
      *id = int( s->reqs.size() ) - 1;
   HYB_API_END
}

int hyb_server_run( hyb_server* s, double timeLimit )
{
   HYB_API_BEGIN
   require( s, "null argument" );
   require( timeLimit > 0, "time limit must be positive" );
   runServer( *s, timeLimit );
   HYB_API_END
}

int hyb_server_result( const hyb_server* s, int id, hyb_request_result* out )
{
   HYB_API_BEGIN
   require( s && out, "null argument" );
   require( id >= 0 && id < int( s->reqs.size() ), "unknown request id" );
   const ServeRequest& r = s->reqs[id];
   require( r.state == kDone, "request not finished" );
   out->status          = r.status;
   out->cycles          = r.cycles;
   out->rel_residual    = r.rel;
   out->arrival_s       = r.arrival;
   out->admit_s         = r.tAdmit;
   out->done_s          = r.tDone;
   out->footprint_bytes = r.served;
   HYB_API_END
}

int hyb_server_stats( const hyb_server* s, size_t* peak, int* built, int* graphs )
{
   HYB_API_BEGIN
   require( s, "null argument" );
   if ( peak )
      *peak = s->peak;
   if ( built )
      *built = s->built;
   if ( graphs )
      *graphs = s->graphsCaptured();
   HYB_API_END
}

int hyb_server_batch_stats( const hyb_server* s, int* batches, int* batched_solves )
{
   HYB_API_BEGIN
   require( s, "null argument" );
   if ( batches )
      *batches = s->batches;
   if ( batched_solves )
      *batched_solves = s->batchedSolves;
   HYB_API_END
}

int hyb_server_mesh_bytes( const hyb_server* s, size_t* bytes )
{
   HYB_API_BEGIN
   require( s && bytes, "null argument" );
   size_t sum = 0;
   for ( auto& m : s->meshes )
      sum += m->bytes;
   *bytes = sum;
   HYB_API_END
}

int hyb_rff_features( uint64_t seed, double corrLen, int modes, double* w, double* phase )
{
   HYB_API_BEGIN
   require( w && phase, "null argument" );
   require( corrLen > 0 && modes >= 1 && modes <= 4096, "invalid feature parameters" );
   rffFeatures( seed, corrLen, modes, w, phase );
   HYB_API_END
}

} // extern "C"
