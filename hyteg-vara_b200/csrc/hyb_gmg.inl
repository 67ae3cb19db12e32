// Geometric multigrid: V/W-cycles, the small-level program, graph capture and replay.
// (part of the single translation unit hyb_capi.cu, included inside namespace hyb)

// ---------------------------------------------------------------------------
// Timing tree: the nested stage timers of the reference's solver (waLBerla WcTimingTree
// owned by the PrimitiveStorage; start/stop in GeometricMultigridSolver.hpp:129-233) with
// the same node names and nesting, measured on the device: start and stop record CUDA
// events on the solve's stream, and collect() waits for the last one and adds each pair's
// elapsed time to its node.
// ---------------------------------------------------------------------------
struct TimingNode
{
   std::string                                name;
   TimingNode*                                parent = nullptr;
   std::vector< std::unique_ptr< TimingNode > > kids;
   double                                     total = 0, minT = 0, maxT = 0; // seconds
   long                                       count = 0;
};

struct TimingTree
{
   TimingNode root;
   TimingNode* cur = &root;
   struct Open
   {
      TimingNode* node;
      cudaEvent_t start;
   };
   struct Pending
   {
      TimingNode* node;
      cudaEvent_t start, stop;
   };
   std::vector< Open >        open;
   std::vector< Pending >     pending;
   std::vector< cudaEvent_t > pool;

   TimingTree() = default;
   TimingTree( const TimingTree& ) = delete;
   TimingTree& operator=( const TimingTree& ) = delete;
   ~TimingTree()
   {
      for ( auto& p : pending )
      {
         cudaEventSynchronize( p.stop );
         pool.push_back( p.start );
         pool.push_back( p.stop );
      }
      for ( auto& o : open )
         pool.push_back( o.start );
      for ( cudaEvent_t e : pool )
         cudaEventDestroy( e );
   }
   cudaEvent_t event()
   {
      if ( !pool.empty() )
      {
         cudaEvent_t e = pool.back();
         pool.pop_back();
         return e;
      }
      cudaEvent_t e;
      HYB_CUDA( cudaEventCreate( &e ) );
      return e;
   }
   void start( const std::string& name, cudaStream_t s )
   {
      TimingNode* child = nullptr;
      for ( auto& k : cur->kids )
         if ( k->name == name )
            child = k.get();
      if ( !child )
      {
         cur->kids.push_back( std::make_unique< TimingNode >() );
         child         = cur->kids.back().get();
         child->name   = name;
         child->parent = cur;
      }
      const cudaEvent_t e = event();
      HYB_CUDA( cudaEventRecord( e, s ) );
      open.push_back( { child, e } );
      cur = child;
   }
   void stop( const std::string& name, cudaStream_t s )
   {
      require( !open.empty() && open.back().node->name == name, "timing tree: stop of a timer that is not open" );
      const cudaEvent_t e = event();
      HYB_CUDA( cudaEventRecord( e, s ) );
      pending.push_back( { open.back().node, open.back().start, e } );
      open.pop_back();
      cur = cur->parent;
   }
   // wait for the recorded events and add their intervals to the nodes
   void collect()
   {
      if ( pending.empty() )
         return;
      HYB_CUDA( cudaEventSynchronize( pending.back().stop ) );
      for ( auto& p : pending )
      {
         HYB_CUDA( cudaEventSynchronize( p.stop ) ); // events of other streams complete on their own
         float ms = 0;
         HYB_CUDA( cudaEventElapsedTime( &ms, p.start, p.stop ) );
         const double t = 1e-3 * double( ms );
         TimingNode&  n = *p.node;
         n.minT         = n.count == 0 ? t : std::min( n.minT, t );
         n.maxT         = n.count == 0 ? t : std::max( n.maxT, t );
         n.total += t;
         ++n.count;
         pool.push_back( p.start );
         pool.push_back( p.stop );
      }
      pending.clear();
   }
   void reset()
   {
      require( open.empty(), "timing tree: reset while a timer is open" );
      collect();
      root.kids.clear();
      cur = &root;
   }
   // {"<name>": {"total": s, "average": s, "min": s, "max": s, "count": n, "children": {...}}, ...}
   static void json( const TimingNode& n, std::string& out )
   {
      out += "{";
      for ( size_t i = 0; i < n.kids.size(); ++i )
      {
         const TimingNode& k = *n.kids[i];
         char              buf[256];
         std::snprintf( buf, sizeof( buf ), "\"total\": %.9g, \"average\": %.9g, \"min\": %.9g, \"max\": %.9g, \"count\": %ld",
                        k.total, k.count ? k.total / double( k.count ) : 0.0, k.minT, k.maxT, k.count );
         out += ( i ? ", \"" : "\"" ) + k.name + "\": {" + buf + ", \"children\": ";
         json( k, out );
         out += "}";
      }
      out += "}";
   }
};

// ---------------------------------------------------------------------------
// Geometric multigrid (GeometricMultigridSolver.hpp:136-235)
// ---------------------------------------------------------------------------
struct Gmg
{
   Storage*  st;
   Operator* op;
   int       minL, maxL, pre, post, smoother, coarseMaxIter;
   int       cycleType = HYB_CYCLE_V;
   double    relax, coarseTol;
   std::unique_ptr< Function > tmp64;         // gmg_tmp
   std::unique_ptr< Function > x32, b32, t32; // FP32 inner hierarchy (mixed precision)
   std::unique_ptr< Function > r64;           // FP64 residual (mixed precision)
   std::unique_ptr< Function > cx64, cb64;    // FP64 coarse-solve copies of the FP32 hierarchy
   std::vector< double >       cheb;          // Chebyshev smoother: omega_0 .. omega_{order-1}
   std::unique_ptr< Function > inv64, inv32;  // Chebyshev smoother: diag(A)^-1 per level
   std::unique_ptr< Function > ch64, ch32;    // Chebyshev smoother: second temporary
   DevBuf< char >              sorCoef;       // reference-order SOR: face couplings
   CgScratch                   cg;
   // reduction scratch of this solver, so that solvers sharing a storage can run on
   // different streams at the same time: scalars[0] = ||r||^2, scalars[1] = ||b||^2
   DevBuf< double >            partial, scalars;
   double*                     hostScalar = nullptr; // pinned, 2 doubles
   // Levels <= progTop of a V-cycle run as one program-kernel launch (-1: none), with one
   // recorded phase list per (x, b, compute type, top level).
   int progTop = -1;
   struct Program
   {
      const void*     x;
      const void*     b;
      int             dtype, top, n;
      DevBuf< Phase > phases;
   };
   std::vector< std::unique_ptr< Program > > programs;
   // whole-solve programs for k_solve_batch (ensureSolveProgram), keyed by (x, b, level =
   // top, step kind in dtype)
   std::vector< std::unique_ptr< Program > > solvePrograms;
   cudaStream_t                cap = nullptr; // capture stream
   // captured graphs keyed by (x, b, level, kind)
   struct G
   {
      const void* x;
      const void* b;
      int         level, kind;
      cudaGraphExec_t exec;
      long long       kernels; // kernel launches captured in the graph
   };
   std::vector< G > graphs;
   // device-iterated solves (runSolveLoop): one graph per (x, b, level, step kind), and the
   // stopping-test state they share (SolveCtl, device and pinned host copy)
   std::vector< G > loops;
   DevBuf< SolveCtl > ctl;
   SolveCtl*          hostCtl = nullptr;
   // stage timers (hyb_gmg_set_timing): while on, solves run launch by launch, without
   // graphs or the program kernel, and every stage records device events
   bool       timing = false;
   TimingTree tt;
   void tstart( const std::string& name, cudaStream_t s )
   {
      if ( timing )
         tt.start( name, s );
   }
   void tstop( const std::string& name, cudaStream_t s )
   {
      if ( timing )
         tt.stop( name, s );
   }

   ~Gmg()
   {
      for ( auto& g : graphs )
         cudaGraphExecDestroy( g.exec );
      for ( auto& g : loops )
         cudaGraphExecDestroy( g.exec );
      if ( hostCtl )
         cudaFreeHost( hostCtl );
      if ( cap )
         cudaStreamDestroy( cap );
      if ( hostScalar )
         cudaFreeHost( hostScalar );
   }
};

constexpr int kGmgFlag = HYB_INNER | HYB_NEUMANN;

template < typename T >
void smooth( Gmg& g, int l, T* x, const T* b, T* scratch, cudaStream_t stream )
{
   if ( g.smoother == HYB_SMOOTHER_SOR )
      launchSor< T >( *g.op, l, x, b, T( g.relax ), kGmgFlag, stream );
   else if ( g.smoother == HYB_SMOOTHER_SYMMETRIC_SOR )
   {
      // SymmetricSORSmoother::solve (SymmetricSORSmoother.hpp:38-57): forward, then backwards
      launchSor< T >( *g.op, l, x, b, T( g.relax ), kGmgFlag, stream );
      launchSor< T >( *g.op, l, x, b, T( g.relax ), kGmgFlag, stream, true );
   }
   else if ( g.smoother == HYB_SMOOTHER_SOR_REFERENCE_ORDER || g.smoother == HYB_SMOOTHER_SYMMETRIC_SOR_REFERENCE_ORDER )
   {
      // the reference's own sweep order; scratch (the solver's residual vector) holds the
      // start-of-sweep snapshot
      T* coef = reinterpret_cast< T* >( g.sorCoef.p );
      launchSorReference< T >( *g.op, l, x, b, T( g.relax ), kGmgFlag, scratch, coef, stream, false );
      if ( g.smoother == HYB_SMOOTHER_SYMMETRIC_SOR_REFERENCE_ORDER )
         launchSorReference< T >( *g.op, l, x, b, T( g.relax ), kGmgFlag, scratch, coef, stream, true );
   }
   else if ( g.smoother == HYB_SMOOTHER_CHEBYSHEV )
   {
      // ChebyshevSmoother::solve (ChebyshevSmoother.hpp:49-96): t = D^-1 (b - A x), x += w_0 t,
      // then t = D^-1 A t, x += w_k t. scratch (the solver's residual vector) and the second
      // temporary are only written on Inner|Neumann DoFs, so they hold 0 elsewhere.
      const bool      f64 = std::is_same< T, double >::value;
      const T*        inv = ( f64 ? g.inv64 : g.inv32 )->template ptr< T >( l );
      T*              t   = scratch;
      T*              t2  = ( f64 ? g.ch64 : g.ch32 )->template ptr< T >( l );
      launchApply< T >( *g.op, l, x, t, b, kGmgFlag, kResidual, stream );
      launchChebUpdate< T >( *g.st, l, inv, t, x, T( g.cheb[0] ), stream );
      for ( size_t k = 1; k < g.cheb.size(); ++k )
      {
         launchApply< T >( *g.op, l, t, t2, nullptr, kGmgFlag, kReplace, stream );
         launchChebUpdate< T >( *g.st, l, inv, t2, x, T( g.cheb[k] ), stream );
         std::swap( t, t2 );
      }
   }
   else
   {
      // Jacobi needs the old iterate: scratch = x, then x = scratch + relax D^-1 (b - A scratch)
      HYB_CUDA( cudaMemcpyAsync( scratch, x, size_t( g.st->td.nC ) * g.st->L( l ).dev.stride * sizeof( T ),
                                 cudaMemcpyDeviceToDevice, stream ) );
      launchJacobi< T >( *g.op, l, scratch, x, b, T( g.relax ), kGmgFlag, stream );
   }
}

// coarse solve: FP64 CG; an FP32 hierarchy is solved through FP64 copies
void coarseSolve( Gmg& g, double* x, const double* b, cudaStream_t stream )
{
   launchCg( *g.op, g.minL, x, b, g.cg, g.coarseTol, g.coarseMaxIter, stream );
}
void coarseSolve( Gmg& g, float* x, const float* b, cudaStream_t stream )
{
   const int l = g.minL;
   launchConvert< double, float >( *g.st, l, g.cx64->ptr< double >( l ), x, stream );
   launchConvert< double, float >( *g.st, l, g.cb64->ptr< double >( l ), b, stream );
   launchCg( *g.op, l, g.cx64->ptr< double >( l ), g.cb64->ptr< double >( l ), g.cg, g.coarseTol, g.coarseMaxIter, stream );
   launchConvert< float, double >( *g.st, l, x, g.cx64->ptr< double >( l ), stream );
}

// ---------------------------------------------------------------------------
// Program-kernel V-cycle for the small levels: the phases mirror vcycle() below, launch
// for launch, with each launch's grid as the phase's virtual grid.
// ---------------------------------------------------------------------------
// levels whose slabs hold at most this many points (all cells) run in the program kernel;
// HYB_PROGRAM_MAX_POINTS overrides it (0: never)
constexpr long kProgramMaxPoints = 4096;

struct PhaseList
{
   const Gmg&           g;
   std::vector< Phase > ph;

   // one thread block runs the program: a phase has one virtual block for its cell-interior
   // loop (if the launch it replaces has one) and one for its surface or flat loop
   Phase& add( int kind, int level, int blocks, int cellBlocks )
   {
      Phase P{};
      P.kind       = kind;
      P.level      = level;
      P.cellBlocks = cellBlocks > 0 ? 1 : 0;
      P.blocks     = std::max( P.cellBlocks + ( blocks > cellBlocks ? 1 : 0 ), 1 );
      P.op32       = g.op->dev< float >( level );
      P.op64       = g.op->dev< double >( level );
      ph.push_back( P );
      return ph.back();
   }
   long slabElems( int l ) const { return long( g.st->td.nC ) * g.st->L( l ).dev.stride; }
   // the row table of level l for the passes of this (constant) operator, built on first use
   const RowTables* rows( int l ) const
   {
      const RowTables* R = ensureRows( *g.st, l );
      return R && R->full ? R : nullptr;
   }
   int  flatBlocks( long n ) const
   {
      return int( std::min< long >( ( n + 127 ) / 128, long( g.st->numSMs ) * 8 ) );
   }

   template < typename T >
   void smooth( int l, T* x, const T* b, T* scratch )
   {
      const Storage& s = *g.st;
      const auto&    L = s.L( l );
      if ( g.smoother == HYB_SMOOTHER_SOR || g.smoother == HYB_SMOOTHER_SYMMETRIC_SOR )
      {
         auto iface = [&]( int c ) {
            const int* co    = &L.colourOff[4 * c];
            const long lanes = bdryLaneCount( co[1], co[2], co[3] );
            if ( lanes == 0 )
               return;
            const int32_t* list = L.colourList.p + co[0];
            Phase&         P    = add( kPhSorIface, l, int( std::min< long >( ( lanes + 127 ) / 128, long( s.numSMs ) * 8 ) ), 0 );
            P.p0                = x;
            P.p1                = const_cast< T* >( b );
            P.relax             = g.relax;
            P.flag              = kGmgFlag;
            P.bl                = BdryLists{ list, list + co[1], list + co[1] + co[2], co[1], co[2], co[3] };
            if ( const RowTables* R = rows( l ) )
            {
               const long b1 = long( co[1] ) * 32, b2 = b1 + ( long( co[2] ) * 8 + 31 ) / 32 * 32;
               P.rp          = RowPass{ R->iface.p + R->ifaceOff[size_t( c )], lanes, b1, b2, lanes };
               P.blocks      = 1;
               P.cellBlocks  = 0;
            }
         };
         auto interior = [&]( int c ) {
            const int count = L.dev.ptsOff[c + 1] - L.dev.ptsOff[c];
            if ( count == 0 )
               return;
            Phase& P = add( kPhSorInterior, l, L.colourBlocks, L.colourBlocks );
            P.p0     = x;
            P.p1     = const_cast< T* >( b );
            P.relax  = g.relax;
            P.a0     = c;
            P.a1     = L.dev.ptsOff[c];
            P.a2     = count;
            if ( const RowTables* R = rows( l ) )
            {
               const long n = long( s.td.nC ) * count;
               P.rp         = RowPass{ R->interior.p + long( s.td.nC ) * L.dev.ptsOff[c], n, 0, 0, 0 };
               P.blocks     = 1;
               P.cellBlocks = 0;
            }
         };
         for ( int c = 0; c < s.td.m; ++c )
            iface( c );
         for ( int c = 0; c < kInteriorColours; ++c )
            interior( c );
         if ( g.smoother == HYB_SMOOTHER_SYMMETRIC_SOR )
         {
            for ( int c = kInteriorColours - 1; c >= 0; --c )
               interior( c );
            for ( int c = s.td.m - 1; c >= 0; --c )
               iface( c );
         }
      }
      else
      {
         Phase& C = add( kPhCopy, l, flatBlocks( slabElems( l ) ), 0 );
         C.p0     = scratch;
         C.p1     = x;
         C.n      = slabElems( l );
         const int nc = L.dev.nPts > 0 ? L.ptsBlocks : 0;
         Phase&    P  = add( kPhJacobi, l, nc + ( L.dev.nBdry > 0 ? L.bdryBlocks : 0 ), nc );
         P.p0         = scratch;
         P.p1         = x;
         P.p2         = const_cast< T* >( b );
         P.relax      = g.relax;
         P.flag       = kGmgFlag;
      }
   }

   void cg( int l, double* x, const double* b )
   {
      Phase& P = add( kPhCg, l, 1, 0 );
      P.p0     = x;
      P.p1     = const_cast< double* >( b );
      P.p2     = g.cg.r->ptr< double >( l );
      P.p3     = g.cg.p->ptr< double >( l );
      P.p4     = g.cg.ap->ptr< double >( l );
      P.status = g.cg.status.p;
      P.relax  = g.coarseTol;
      P.a0     = g.coarseMaxIter;
      P.rp     = rowPassAll( rows( l ) );
   }

   // phases of a whole solve (k_solve_batch)
   void residual64( int l, double* x, double* r, const double* b )
   {
      const auto& L  = g.st->L( l );
      const int   nc = L.dev.nPts > 0 ? L.ptsBlocks : 0;
      Phase&      P  = add( kPhResidual, l, nc + ( L.dev.nBdry > 0 ? L.bdryBlocks : 0 ), nc );
      P.p0           = x;
      P.p1           = r;
      P.p2           = const_cast< double* >( b );
      P.flag         = kGmgFlag;
      if ( const RowTables* R = rows( l ) )
      {
         P.rp         = rowPassAll( R );
         P.blocks     = 1;
         P.cellBlocks = 0;
      }
   }
   void dot( int l, const double* a, const double* b, float* cvt, int slot )
   {
      Phase& P = add( kPhDot, l, 1, 0 );
      P.p0     = const_cast< double* >( a );
      P.p1     = const_cast< double* >( b );
      P.p2     = cvt;
      P.flag   = kGmgFlag;
      P.a0     = slot;
   }
   void zero32( int l, float* p )
   {
      Phase& P = add( kPhZero, l, flatBlocks( slabElems( l ) ), 0 );
      P.p0     = p;
      P.n      = slabElems( l );
      P.dtype  = HYB_F32;
   }
   void addCorr( int l, double* x, const float* e )
   {
      Phase& P = add( kPhAddCorr, l, 1, 0 );
      P.p0     = x;
      P.p1     = const_cast< float* >( e );
      P.flag   = kGmgFlag;
   }
   void ctl( SolveCtl* c, int loopStart, int init )
   {
      Phase& P = add( kPhCtl, 0, 1, 0 );
      P.p0     = c;
      P.a0     = loopStart;
      P.a1     = init;
   }

   void coarse( double* x, const double* b ) { cg( g.minL, x, b ); }
   void coarse( float* x, const float* b )
   {
      const int  l = g.minL;
      const long n = slabElems( l );
      Phase&     A = add( kPhToF64, l, flatBlocks( n ), 0 );
      A.p0         = g.cx64->ptr< double >( l );
      A.p1         = x;
      A.n          = n;
      Phase& B     = add( kPhToF64, l, flatBlocks( n ), 0 );
      B.p0         = g.cb64->ptr< double >( l );
      B.p1         = const_cast< float* >( b );
      B.n          = n;
      cg( l, g.cx64->ptr< double >( l ), g.cb64->ptr< double >( l ) );
      Phase& C = add( kPhToF32, l, flatBlocks( n ), 0 );
      C.p0     = x;
      C.p1     = g.cx64->ptr< double >( l );
      C.n      = n;
   }

   template < typename T >
   void vcycle( Function& x, Function& b, Function& tmp, int l )
   {
      if ( l == g.minL )
      {
         coarse( x.ptr< T >( l ), b.ptr< T >( l ) );
         return;
      }
      const Storage& s = *g.st;
      for ( int i = 0; i < g.pre; ++i )
         smooth< T >( l, x.ptr< T >( l ), b.ptr< T >( l ), tmp.ptr< T >( l ) );
      {
         const auto& L  = s.L( l );
         const int   nc = L.dev.nPts > 0 ? L.ptsBlocks : 0;
         Phase&      P  = add( kPhResidual, l, nc + ( L.dev.nBdry > 0 ? L.bdryBlocks : 0 ), nc );
         P.p0           = x.ptr< T >( l );
         P.p1           = tmp.ptr< T >( l );
         P.p2           = b.ptr< T >( l );
         P.flag         = kGmgFlag;
         if ( const RowTables* R = rows( l ) )
         {
            P.rp         = rowPassAll( R );
            P.blocks     = 1;
            P.cellBlocks = 0;
         }
      }
      {
         const auto& C  = s.L( l - 1 );
         const int   nc = C.dev.nSeg > 0 ? C.cellBlocks : 0;
         Phase&      P  = add( kPhRestrict, l - 1, nc + ( C.dev.nBdry > 0 ? C.bdryBlocks : 0 ), nc );
         P.p0           = tmp.ptr< T >( l );
         P.p1           = b.ptr< T >( l - 1 );
         P.flag         = kGmgFlag;
      }
      {
         Phase& P = add( kPhZero, l - 1, flatBlocks( slabElems( l - 1 ) ), 0 );
         P.p0     = x.ptr< T >( l - 1 );
         P.n      = slabElems( l - 1 );
      }
      vcycle< T >( x, b, tmp, l - 1 );
      if ( g.cycleType == HYB_CYCLE_W )
         vcycle< T >( x, b, tmp, l - 1 );
      {
         const auto& F  = s.L( l );
         const int   nc = F.dev.nPts > 0 ? F.ptsBlocks : 0;
         Phase&      P  = add( kPhProlongAdd, l, nc + ( F.dev.nBdry > 0 ? F.bdryBlocks : 0 ), nc );
         P.p0           = x.ptr< T >( l - 1 );
         P.p1           = x.ptr< T >( l );
         P.flag         = kGmgFlag;
      }
      for ( int i = 0; i < g.post; ++i )
         smooth< T >( l, x.ptr< T >( l ), b.ptr< T >( l ), tmp.ptr< T >( l ) );
   }
};

// Record (once, outside any stream capture) the program of the sub-cycle at level `top`
// for the V-cycle on (x, b, tmp) in type T.
template < typename T >
void ensureProgram( Gmg& g, Function& x, Function& b, Function& tmp, int top )
{
   const int dtype = std::is_same< T, double >::value ? HYB_F64 : HYB_F32;
   for ( auto& p : g.programs )
      if ( p->x == &x && p->b == &b && p->dtype == dtype && p->top == top )
         return;
   PhaseList pl{ g, {} };
   pl.vcycle< T >( x, b, tmp, top );
   auto prog   = std::make_unique< Gmg::Program >();
   prog->x     = &x;
   prog->b     = &b;
   prog->dtype = dtype;
   prog->top   = top;
   prog->n     = int( pl.ph.size() );
   prog->phases.upload( pl.ph );
   g.programs.push_back( std::move( prog ) );
}

template < typename T >
void launchProgram( Gmg& g, Function& x, Function& b, int top, cudaStream_t stream )
{
   const int           dtype = std::is_same< T, double >::value ? HYB_F64 : HYB_F32;
   const Gmg::Program* prog  = nullptr;
   for ( auto& p : g.programs )
      if ( p->x == &x && p->b == &b && p->dtype == dtype && p->top == top )
         prog = p.get();
   require( prog != nullptr, "program of the coarse V-cycle was not recorded" );
   const Phase* ph  = prog->phases.p;
   const auto*  lt  = (const LevelDev*) g.st->lvTable.p;
   const int    nLv = int( g.st->lvTable.n );
   require( varKind( *g.op ) != 2, "the program kernel does not take coefficients at quadrature points" );
   if ( g.op->variable )
      pdlLaunch( k_program< T, true >, dim3( 1 ), dim3( kProgramThreads ), 0, stream, g.st->td, lt, ph, prog->n, nLv );
   else
      pdlLaunch( k_program< T, false >, dim3( 1 ), dim3( kProgramThreads ), 0, stream, g.st->td, lt, ph, prog->n, nLv );
   HYB_CHECK_LAUNCH();
}

template < typename T >
void vcycle( Gmg& g, Function& x, Function& b, Function& tmp, int l, cudaStream_t stream )
{
   if ( l <= g.progTop && !g.timing )
   {
      launchProgram< T >( g, x, b, l, stream );
      return;
   }
   const std::string lname = "Level " + std::to_string( l );
   if ( l == g.minL )
   {
      g.tstart( lname, stream );
      g.tstart( "Coarse Grid Solver", stream );
      coarseSolve( g, x.ptr< T >( l ), b.ptr< T >( l ), stream );
      g.tstop( "Coarse Grid Solver", stream );
      g.tstop( lname, stream );
      return;
   }
   g.tstart( lname, stream );
   for ( int i = 0; i < g.pre; ++i )
   {
      g.tstart( "Smoother", stream );
      smooth< T >( g, l, x.ptr< T >( l ), b.ptr< T >( l ), tmp.ptr< T >( l ), stream );
      g.tstop( "Smoother", stream );
   }
   // tmp = b - A x ; restricted straight into b on the coarser level (b.assign(tmp) on flag)
   launchApply< T >( *g.op, l, x.ptr< T >( l ), tmp.ptr< T >( l ), b.ptr< T >( l ), kGmgFlag, kResidual, stream );
   g.tstart( "Restriction", stream );
   launchRestrict< T >( *g.st, l, tmp.ptr< T >( l ), b.ptr< T >( l - 1 ), kGmgFlag, stream );
   g.tstop( "Restriction", stream );
   HYB_CUDA( cudaMemsetAsync( x.ptr< T >( l - 1 ), 0, x.levelBytes( l - 1 ), stream ) ); // x.interpolate(0, l-1)
   g.tstop( lname, stream );
   vcycle< T >( g, x, b, tmp, l - 1, stream );
   if ( g.cycleType == HYB_CYCLE_W ) // GeometricMultigridSolver.hpp:201-204
      vcycle< T >( g, x, b, tmp, l - 1, stream );
   g.tstart( lname, stream );
   g.tstart( "Prolongation", stream );
   launchProlongate< T >( *g.st, l - 1, x.ptr< T >( l - 1 ), x.ptr< T >( l ), kGmgFlag, true, stream );
   g.tstop( "Prolongation", stream );
   for ( int i = 0; i < g.post; ++i )
   {
      g.tstart( "Smoother", stream );
      smooth< T >( g, l, x.ptr< T >( l ), b.ptr< T >( l ), tmp.ptr< T >( l ), stream );
      g.tstop( "Smoother", stream );
   }
   g.tstop( lname, stream );
}

// Graph-captured work units.
enum GraphKind : int
{
   kCycle64      = 0, // one FP64 V-cycle
   kCycle64Norm  = 1, // FP64 V-cycle, then r = b - A x and ||r||^2 into scalar slot 0
   kMixedStep    = 2, // FP32 V-cycle on A e = r (r from the previous step), x += e, new r and ||r||^2
   kNorm64       = 3, // r = b - A x into gmg_tmp and ||r||^2
   kNormMixed    = 4, // r = b - A x into the FP64 residual of the mixed solver and ||r||^2
   kFmg64        = 8, // full multigrid, kFmg64 + c: c FP64 V-cycles per level (1 <= c <= 8)
};

void enqueue( Gmg& g, Function& x, Function& b, int l, int kind, cudaStream_t s )
{
   if ( kind == kCycle64 || kind == kCycle64Norm )
   {
      g.tstart( "Geometric Multigrid Solver", s );
      vcycle< double >( g, x, b, *g.tmp64, l, s );
      g.tstop( "Geometric Multigrid Solver", s );
   }
   if ( kind == kMixedStep )
   {
      // FP32 V-cycle on the residual equation (mixedPrecisionIterativeRefinement.cpp:162-171);
      // the FP32 right-hand side was written with the previous residual's norm (below)
      HYB_CUDA( cudaMemsetAsync( g.x32->ptr< float >( l ), 0, g.x32->levelBytes( l ), s ) );
      g.tstart( "Geometric Multigrid Solver", s );
      vcycle< float >( g, *g.x32, *g.b32, *g.t32, l, s );
      g.tstop( "Geometric Multigrid Solver", s );
      launchAddCorrection< float >( *g.st, l, x.ptr< double >( l ), g.x32->ptr< float >( l ), kGmgFlag, s );
   }
   if ( kind > kFmg64 && kind <= kFmg64 + 8 )
   {
      // FullMultigridSolver::solve (FullMultigridSolver.hpp:51-75) with linear FMG
      // prolongation on inner and Neumann DoFs
      for ( int lc = g.minL; lc <= l; ++lc )
      {
         for ( int c = 0; c < kind - kFmg64; ++c )
         {
            g.tstart( "Geometric Multigrid Solver", s );
            vcycle< double >( g, x, b, *g.tmp64, lc, s );
            g.tstop( "Geometric Multigrid Solver", s );
         }
         if ( lc < l )
            launchProlongate< double >( *g.st, lc, x.ptr< double >( lc ), x.ptr< double >( lc + 1 ), kGmgFlag, false, s );
      }
      return;
   }
   if ( kind != kCycle64 )
   {
      const bool mixed = kind == kMixedStep || kind == kNormMixed;
      float*     cvt   = mixed ? g.b32->ptr< float >( l ) : nullptr;
      const RowTables* R = rowsIf( *g.st, l );
      // ||r||^2 in the residual pass itself (r is not stored); for the mixed solver the same
      // pass writes the next FP32 right-hand side
      if ( !( R && R->full ) && launchResidualNorm< double >( *g.op, l, x.ptr< double >( l ), b.ptr< double >( l ), kGmgFlag,
                                                              g.partial.p, g.partial.n, g.scalars.p, cvt, s ) )
         return;
      Function& r = mixed ? *g.r64 : *g.tmp64;
      launchApply< double >( *g.op, l, x.ptr< double >( l ), r.ptr< double >( l ), b.ptr< double >( l ), kGmgFlag, kResidual, s );
      launchDot< double >( *g.st, l, r.ptr< double >( l ), r.ptr< double >( l ), kGmgFlag, g.partial.p, g.scalars.p, s, cvt );
   }
}

// everything a captured graph needs is allocated before capture begins
// the Chebyshev smoother's inverse diagonals and temporaries for the hierarchies in use
void ensureChebyshev( Gmg& g )
{
   if ( g.smoother != HYB_SMOOTHER_CHEBYSHEV )
      return;
   require( !g.cheb.empty(), "the Chebyshev smoother needs its coefficients (hyb_gmg_setup_chebyshev)" );
   auto fill = [&]( std::unique_ptr< Function >& inv, std::unique_ptr< Function >& t2, int dtype ) {
      if ( inv )
         return;
      inv.reset( makeFunction( g.st, g.minL, g.maxL, dtype ) );
      t2.reset( makeFunction( g.st, g.minL, g.maxL, dtype ) );
      for ( int l = g.minL; l <= g.maxL; ++l )
         if ( dtype == HYB_F64 )
            launchInvDiag< double >( *g.op, l, t2->ptr< double >( l ), inv->ptr< double >( l ), nullptr );
         else
            launchInvDiag< float >( *g.op, l, t2->ptr< float >( l ), inv->ptr< float >( l ), nullptr );
      HYB_CUDA( cudaDeviceSynchronize() );
   };
   fill( g.inv64, g.ch64, HYB_F64 );
   if ( g.x32 )
      fill( g.inv32, g.ch32, HYB_F32 );
}

void prepare( Gmg& g )
{
   ensureChebyshev( g );
   if ( g.smoother == HYB_SMOOTHER_SOR_REFERENCE_ORDER || g.smoother == HYB_SMOOTHER_SYMMETRIC_SOR_REFERENCE_ORDER )
   {
      // tables, kernel attributes and this solver's own face-coupling scratch (FP64 sizes
      // cover FP32), all before any graph is captured
      size_t n = 0;
      for ( int l = g.minL; l <= g.maxL; ++l )
      {
         sorRefPrepare< double >( *g.st, l );
         sorRefPrepare< float >( *g.st, l );
         n = std::max( n, sorRefCoefElems( *g.st, l ) );
      }
      if ( g.sorCoef.n < std::max< size_t >( n, 1 ) * sizeof( double ) )
         g.sorCoef.alloc( std::max< size_t >( n, 1 ) * sizeof( double ) );
   }
   for ( int l = g.minL; l <= g.maxL; ++l )
      ensureRows( *g.st, l );
   if ( !g.cg.r )
   {
      g.cg.r.reset( makeFunction( g.st, g.minL, g.minL, HYB_F64 ) );
      g.cg.p.reset( makeFunction( g.st, g.minL, g.minL, HYB_F64 ) );
      g.cg.ap.reset( makeFunction( g.st, g.minL, g.minL, HYB_F64 ) );
      g.cg.status.alloc( 4 );
   }
}

void initGmg( Gmg& g, Storage* s, Operator* op, int minL, int maxL, int pre, int post, double relax, int smoother,
              double coarseTol, int coarseMaxIter )
{
   g.st            = s;
   g.op            = op;
   g.minL          = minL;
   g.maxL          = maxL;
   g.pre           = pre;
   g.post          = post;
   g.relax         = relax;
   g.smoother      = smoother;
   g.coarseTol     = coarseTol;
   g.coarseMaxIter = coarseMaxIter;
   g.tmp64.reset( makeFunction( s, minL, maxL, HYB_F64 ) );
   g.partial.alloc( s->partial.n );
   g.scalars.alloc( 2 );
   HYB_CUDA( cudaMallocHost( &g.hostScalar, 2 * sizeof( double ) ) );
   long maxPoints = kProgramMaxPoints;
   if ( const char* e = std::getenv( "HYB_PROGRAM_MAX_POINTS" ) )
      maxPoints = std::atol( e );
   g.progTop = -1;
   for ( int l = minL; l <= maxL; ++l )
      if ( long( s->td.nC ) * s->L( l ).dev.stride <= maxPoints )
         g.progTop = l;
   if ( smoother == HYB_SMOOTHER_CHEBYSHEV || smoother == HYB_SMOOTHER_SOR_REFERENCE_ORDER ||
        smoother == HYB_SMOOTHER_SYMMETRIC_SOR_REFERENCE_ORDER )
      g.progTop = -1; // the program kernel has no Chebyshev or reference-order SOR phases
   if ( op->blend )
      g.progTop = -1; // blending operators run every level as row-pass launches
   if ( varKind( *op ) == 2 )
      g.progTop = -1; // the program kernel is built for nodal coefficients only
}


// the FP32 hierarchy and FP64 residual of the mixed-precision solver
void ensureMixed( Gmg& g )
{
   if ( g.x32 )
      return;
   Storage* s = g.st;
   g.x32.reset( makeFunction( s, g.minL, g.maxL, HYB_F32 ) );
   g.b32.reset( makeFunction( s, g.minL, g.maxL, HYB_F32 ) );
   g.t32.reset( makeFunction( s, g.minL, g.maxL, HYB_F32 ) );
   g.r64.reset( makeFunction( s, g.minL, g.maxL, HYB_F64 ) );
   g.cx64.reset( makeFunction( s, g.minL, g.minL, HYB_F64 ) );
   g.cb64.reset( makeFunction( s, g.minL, g.minL, HYB_F64 ) );
}

void runGraph( Gmg& g, Function& x, Function& b, int l, int kind, cudaStream_t stream )
{
   if ( g.timing )
   {
      // timed: launch by launch, so that the stage events sit between the stages' kernels
      prepare( g );
      enqueue( g, x, b, l, kind, stream );
      return;
   }
   for ( auto& G : g.graphs )
      if ( G.x == &x && G.b == &b && G.level == l && G.kind == kind )
      {
         HYB_CUDA( cudaGraphLaunch( G.exec, stream ) );
         g_launches.fetch_add( G.kernels, std::memory_order_relaxed );
         return;
      }
   prepare( g );
   if ( g.progTop >= g.minL )
   {
      const int top = std::min( l, g.progTop );
      if ( kind == kCycle64 || kind == kCycle64Norm )
         ensureProgram< double >( g, x, b, *g.tmp64, top );
      if ( kind > kFmg64 && kind <= kFmg64 + 8 )
         for ( int t = g.minL; t <= top; ++t )
            ensureProgram< double >( g, x, b, *g.tmp64, t );
      if ( kind == kMixedStep )
         ensureProgram< float >( g, *g.x32, *g.b32, *g.t32, top );
   }
   if ( !g.cap )
      HYB_CUDA( cudaStreamCreateWithFlags( &g.cap, cudaStreamNonBlocking ) );
   // make the capture stream wait for prior work on the caller's stream
   cudaEvent_t ev;
   HYB_CUDA( cudaEventCreateWithFlags( &ev, cudaEventDisableTiming ) );
   HYB_CUDA( cudaEventRecord( ev, stream ) );
   HYB_CUDA( cudaStreamWaitEvent( g.cap, ev, 0 ) );
   HYB_CUDA( cudaStreamSynchronize( g.cap ) );
   HYB_CUDA( cudaEventDestroy( ev ) );
   cudaGraph_t     graph = nullptr;
   const long long before = g_launches.load();
   HYB_CUDA( cudaStreamBeginCapture( g.cap, cudaStreamCaptureModeThreadLocal ) );
   try
   {
      enqueue( g, x, b, l, kind, g.cap );
   }
   catch ( ... )
   {
      cudaStreamEndCapture( g.cap, &graph );
      if ( graph )
         cudaGraphDestroy( graph );
      throw;
   }
   HYB_CUDA( cudaStreamEndCapture( g.cap, &graph ) );
   const long long captured = g_launches.load() - before;
   g_launches.fetch_sub( captured ); // counted when the graph runs
   cudaGraphExec_t exec;
   HYB_CUDA( cudaGraphInstantiate( &exec, graph, 0 ) );
   HYB_CUDA( cudaGraphDestroy( graph ) );
   g.graphs.push_back( { &x, &b, l, kind, exec, captured } );
   HYB_CUDA( cudaGraphLaunch( exec, stream ) );
   g_launches.fetch_add( captured );
}

// A whole solve as ONE graph launch: while ||b - A x|| / ||b|| > tol (and fewer than
// maxCycles steps ran), run the step `kind` (kCycle64Norm: an FP64 V-cycle; kMixedStep: an
// FP32 V-cycle with FP64 refinement), each followed by the device-side stopping test
// (k_solve_ctl) that sets the condition of the graph's WHILE node -- no host round trip
// per cycle. Before it, the residual norm of the start iterate must be in scalars[0] and
// ||b||^2 in scalars[1] (the kNorm64 / kNormMixed graphs and a dot product). Afterwards
// g.ctl holds the cycles run and the final relative residual.
void runSolveLoop( Gmg& g, Function& x, Function& b, int l, int kind, double tol, int maxCycles, cudaStream_t stream )
{
   require( kind == kCycle64Norm || kind == kMixedStep, "the solve loop iterates V-cycles or refinement steps" );
   if ( !g.ctl.p )
   {
      g.ctl.alloc( 1 );
      HYB_CUDA( cudaMallocHost( &g.hostCtl, sizeof( SolveCtl ) ) );
   }
   g.hostCtl->tol       = tol;
   g.hostCtl->maxCycles = maxCycles;
   HYB_CUDA( cudaMemcpyAsync( g.ctl.p, g.hostCtl, sizeof( SolveCtl ), cudaMemcpyHostToDevice, stream ) );
   for ( auto& G : g.loops )
      if ( G.x == &x && G.b == &b && G.level == l && G.kind == kind )
      {
         HYB_CUDA( cudaGraphLaunch( G.exec, stream ) );
         return; // (its kernels are counted by the graph's step launches only approximately)
      }
   prepare( g );
   if ( g.progTop >= g.minL )
   {
      const int top = std::min( l, g.progTop );
      if ( kind == kCycle64Norm )
         ensureProgram< double >( g, x, b, *g.tmp64, top );
      else
         ensureProgram< float >( g, *g.x32, *g.b32, *g.t32, top );
   }
   if ( !g.cap )
      HYB_CUDA( cudaStreamCreateWithFlags( &g.cap, cudaStreamNonBlocking ) );
   HYB_CUDA( cudaStreamSynchronize( stream ) ); // the capture stream must not overtake prior work
   cudaGraph_t outer = nullptr;
   HYB_CUDA( cudaGraphCreate( &outer, 0 ) );
   try
   {
      cudaGraphConditionalHandle h;
      HYB_CUDA( cudaGraphConditionalHandleCreate( &h, outer, 0, 0 ) );
      SolveCtl*            c    = g.ctl.p;
      const double*        sc   = g.scalars.p;
      int                  one  = 1;
      void*                ia[] = { &h, &c, &sc, &one };
      cudaKernelNodeParams kp{};
      kp.func         = reinterpret_cast< void* >( k_solve_ctl );
      kp.gridDim      = dim3( 1 );
      kp.blockDim     = dim3( 1 );
      kp.kernelParams = ia;
      cudaGraphNode_t init;
      HYB_CUDA( cudaGraphAddKernelNode( &init, outer, nullptr, 0, &kp ) );
      cudaGraphNodeParams cp{};
      cp.type                = cudaGraphNodeTypeConditional;
      cp.conditional.handle  = h;
      cp.conditional.type    = cudaGraphCondTypeWhile;
      cp.conditional.size    = 1;
      cudaGraphNode_t whileNode;
      HYB_CUDA( cudaGraphAddNode( &whileNode, outer, &init, 1, &cp ) );
      cudaGraph_t body = cp.conditional.phGraph_out[0];
      const long long before = g_launches.load();
      HYB_CUDA( cudaStreamBeginCaptureToGraph( g.cap, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal ) );
      try
      {
         enqueue( g, x, b, l, kind, g.cap );
         k_solve_ctl<<< 1, 1, 0, g.cap >>>( h, c, sc, 0 );
         HYB_CHECK_LAUNCH();
      }
      catch ( ... )
      {
         cudaGraph_t dummy = nullptr;
         cudaStreamEndCapture( g.cap, &dummy );
         throw;
      }
      HYB_CUDA( cudaStreamEndCapture( g.cap, &body ) );
      const long long captured = g_launches.load() - before;
      g_launches.fetch_sub( captured );
      cudaGraphExec_t exec;
      HYB_CUDA( cudaGraphInstantiate( &exec, outer, 0 ) );
      HYB_CUDA( cudaGraphDestroy( outer ) );
      outer = nullptr;
      g.loops.push_back( { &x, &b, l, kind, exec, captured } );
      HYB_CUDA( cudaGraphLaunch( exec, stream ) );
   }
   catch ( ... )
   {
      if ( outer )
         cudaGraphDestroy( outer );
      throw;
   }
}

// Record (once, outside any stream capture) the whole solve of (x, b) at level l as one
// program for k_solve_batch: ||b||^2, the start residual and its norm (with the FP32
// right-hand side for mixed precision), the stopping test, then the loop of V-cycles
// (kCycle64Norm) or refinement steps (kMixedStep: x32 = 0, FP32 V-cycle, x += x32), each
// followed by the residual norm and the test, which jumps back to the loop's start while
// ||r|| / ||b|| > tol and fewer than maxCycles steps ran. The phases mirror enqueue() and
// runSolveLoop() operation for operation; the whole V-cycle must fit the program kernel
// (l <= progTop). Returns the program, whose tolerance and cycle limit sit in g.ctl.
const Gmg::Program* ensureSolveProgram( Gmg& g, Function& x, Function& b, int l, int kind )
{
   require( kind == kCycle64Norm || kind == kMixedStep, "a solve program iterates V-cycles or refinement steps" );
   for ( auto& p : g.solvePrograms )
      if ( p->x == &x && p->b == &b && p->dtype == kind && p->top == l )
         return p.get();
   require( g.progTop >= l && l > g.minL, "a batched solve needs its whole V-cycle in the program kernel" );
   prepare( g );
   if ( !g.ctl.p )
   {
      g.ctl.alloc( 1 );
      HYB_CUDA( cudaMallocHost( &g.hostCtl, sizeof( SolveCtl ) ) );
   }
   const bool mixed = kind == kMixedStep;
   if ( mixed )
      ensureMixed( g );
   Function& r   = mixed ? *g.r64 : *g.tmp64;
   float*    cvt = mixed ? g.b32->ptr< float >( l ) : nullptr;
   PhaseList pl{ g, {} };
   pl.dot( l, b.ptr< double >( l ), b.ptr< double >( l ), nullptr, 1 );
   pl.residual64( l, x.ptr< double >( l ), r.ptr< double >( l ), b.ptr< double >( l ) );
   pl.dot( l, r.ptr< double >( l ), r.ptr< double >( l ), cvt, 0 );
   const size_t init = pl.ph.size();
   pl.ctl( g.ctl.p, 0, 1 );
   const int loopStart = int( pl.ph.size() );
   if ( mixed )
   {
      pl.zero32( l, g.x32->ptr< float >( l ) );
      const size_t c0 = pl.ph.size();
      pl.vcycle< float >( *g.x32, *g.b32, *g.t32, l );
      for ( size_t i = c0; i < pl.ph.size(); ++i )
         pl.ph[i].dtype = HYB_F32;
      pl.addCorr( l, x.ptr< double >( l ), g.x32->ptr< float >( l ) );
   }
   else
      pl.vcycle< double >( x, b, *g.tmp64, l );
   pl.residual64( l, x.ptr< double >( l ), r.ptr< double >( l ), b.ptr< double >( l ) );
   pl.dot( l, r.ptr< double >( l ), r.ptr< double >( l ), cvt, 0 );
   pl.ctl( g.ctl.p, loopStart, 0 );
   pl.ph[init].a0 = loopStart;
   auto prog   = std::make_unique< Gmg::Program >();
   prog->x     = &x;
   prog->b     = &b;
   prog->dtype = kind;
   prog->top   = l;
   prog->n     = int( pl.ph.size() );
   prog->phases.upload( pl.ph );
   g.solvePrograms.push_back( std::move( prog ) );
   return g.solvePrograms.back().get();
}

// Up to kSolveBatchMax solves in one launch of k_solve_batch (one block each); every job's
// SolveCtl must hold its tolerance and cycle limit in stream order before the launch.
constexpr int kSolveBatchMax = 64;
struct SolveBatch
{
   SolveJob job[kSolveBatchMax];
};

template < int VAR >
__global__ void __launch_bounds__( kProgramThreads ) k_solve_batch( const __grid_constant__ SolveBatch batch )
{
   // the job table travels in the launch's parameters, so no buffer outlives the launch
   solveBatchBody< VAR >( batch.job );
}

// The job of one recorded solve program (ensureSolveProgram) of g.
SolveJob solveJob( const Gmg& g, const Gmg::Program& p )
{
   return SolveJob{ g.st->td, (const LevelDev*) g.st->lvTable.p, p.phases.p, int( g.st->lvTable.n ), p.n };
}

// Every job in launches of at most kSolveBatchMax blocks; var selects the operator kind
// (every job of the call must have that kind).
void launchSolveBatch( const std::vector< SolveJob >& jobs, bool var, cudaStream_t stream )
{
   for ( size_t i0 = 0; i0 < jobs.size(); i0 += kSolveBatchMax )
   {
      const int  n = int( std::min< size_t >( kSolveBatchMax, jobs.size() - i0 ) );
      SolveBatch B{};
      for ( int i = 0; i < n; ++i )
         B.job[i] = jobs[i0 + size_t( i )];
      if ( var )
         k_solve_batch< true ><<< n, kProgramThreads, 0, stream >>>( B );
      else
         k_solve_batch< false ><<< n, kProgramThreads, 0, stream >>>( B );
      HYB_CHECK_LAUNCH();
   }
}
