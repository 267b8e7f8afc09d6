/*
 * propagate_gpu.c -- the reference's time loop replaced by the B200 engine,
 * built INTO the reference (test infrastructure; oracle/build_ref.sh links it
 * into the variant vulture_ref_gpu).
 *
 * This is the reference-side binding of the C ABI in include/vgpu.h: the
 * function propagate() of src/simulation.c:136-231 (declared at
 * src/simulation.h:41, called from src/vulture.c:173) with the same name and
 * signature.  It reads the state the reference has built by then -- the
 * grid globals of src/grid.h:60-147, and, through getters appended to copies
 * of pml.c, mur.c, source.c and observer.c, those modules' private state --
 * into a vgpu_problem, runs every step on the GPU, and hands each step's
 * field samples at the observer points back to the reference's own
 * updateObservers() (src/observer.c:620-650).  The observer files are
 * therefore written, and the frequency-domain sums accumulated, by the
 * reference's code, from the engine's samples.
 *
 * Mapped: the bulk grid and its coefficient volumes (the reference's default
 * unindexed, unscaled build), ghost PEC/PMC/periodic faces, UPML regions,
 * first-order Mur faces, field and current-density sources, and ASCII,
 * binary and waveform observers.  Meshes with plane waves, SIBC surfaces or
 * Debye media stop with the reference's error exit: this replacement does not
 * map them (the whole-CLI replacement, vulture-b200, runs them on the same
 * engine).
 *
 * Requires `real` = double (the FP64 oracle variant), so that the samples
 * handed to the reference are the values the CPU loop would compute.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "fdtd_types.h"
#include "grid.h"
#include "simulation.h"
#include "surface.h"
#include "boundary.h"
#include "medium.h"
#include "planewave.h"
#include "sibc.h"
#include "source.h"
#include "observer.h"
#include "waveform.h"
#include "message.h"
#include "timer.h"

#include "vgpu.h"

#ifdef USE_INDEXED_MEDIA
#error "propagate_gpu.c reads the coefficient volumes of the unindexed build"
#endif
#ifdef USE_SCALE_FIELDS
#error "propagate_gpu.c maps the unscaled field build"
#endif

/* Getters appended to the module copies (oracle/propagate_gpu/state_*.inc.c). */
void vrefPmlState( int present[6] , int lim[6][6][6] , real *prof[6][3] );
void vrefMurState( int lim[6][6][6] , real z[6] );
int vrefNumSources( void );
void vrefSource( int q , int *type , int *field , int *isSoft , int flim[6] , WaveformIndex *waveform ,
                 real *size , real *delay );
int vrefNumObservers( void );
void vrefObserver( int q , int *format , int *domain , int *quantity , int gbbox[6] , int step[3] );

static void *xcalloc( size_t n , size_t size )
{
  void *p = calloc( n ? n : 1 , size );
  if( p == NULL )
    message( MSG_ERROR , 0 , "propagate (GPU): out of host memory\n" );
  return p;
}

static void check( int rc , const char *what )
{
  if( rc != VGPU_OK )
    message( MSG_ERROR , 0 , "propagate (GPU): %s failed (%d): %s\n" , what , rc , vgpu_last_error() );
}

void propagate( void )
{
  vgpu_problem p;
  vgpu_engine *engine = NULL;
  int *points = NULL;
  unsigned long numSteps = getNumTimeSteps();
  real dt = getGridTimeStep();

  if( sizeof( real ) != sizeof( double ) )
    message( MSG_ERROR , 0 , "propagate (GPU): this replacement needs real = double\n" );
  if( thereArePlaneWaves() || thereAreSibcSurfaces() || thereAreMedia( MT_DEBYE ) )
    message( MSG_ERROR , 0 , "propagate (GPU): plane waves, SIBC surfaces and Debye media are not mapped by "
             "this replacement\n" );

  memset( &p , 0 , sizeof p );
  p.abi_version = VGPU_ABI_VERSION;
  p.precision = VGPU_FP64;

  /* Grid (src/grid.c:326-454, 583-679). */
  for( int a = 0 ; a < 3 ; a++ ) p.n[a] = numCells[a];
  for( int b = 0 ; b < 6 ; b++ )
  {
    p.gibox[b] = gibox[b];
    p.gobox[b] = gobox[b];
    for( int f = 0 ; f < 6 ; f++ ) p.gfilim[b][f] = gfilim[b][f];
  }
  p.num_steps = numSteps;
  p.dt = dt;
  p.ide[0] = idex; p.ide[1] = idey; p.ide[2] = idez;
  p.idh[0] = idhx; p.idh[1] = idhy; p.idh[2] = idhz;
  /* allocArray keeps a volume's values in one block after its row
   * pointers (src/alloc_array.c:54-141). */
  p.coef[0] = &alphaEx[0][0][0]; p.coef[1] = &alphaEy[0][0][0]; p.coef[2] = &alphaEz[0][0][0];
  p.coef[3] = &betaEx[0][0][0];  p.coef[4] = &betaEy[0][0][0];  p.coef[5] = &betaEz[0][0][0];
  p.coef[6] = &gammaHx[0][0][0]; p.coef[7] = &gammaHy[0][0][0]; p.coef[8] = &gammaHz[0][0][0];

  /* External faces (src/surface.c:569-812) and their absorbing updates. */
  for( int f = XLO ; f <= ZHI ; f++ )
  {
    BoundaryType t = outerSurfaceType( (MeshFace)f );
    p.ghost[f] = t == BT_PEC ? VGPU_GHOST_PEC : t == BT_PMC ? VGPU_GHOST_PMC
               : t == BT_PERIODIC ? VGPU_GHOST_PERIODIC : VGPU_GHOST_NONE;
    p.mur_present[f] = t == BT_MUR;
  }
  {
    real *prof[6][3];
    vrefPmlState( p.pml_present , p.pml_flim , prof );
    for( int a = 0 ; a < 3 ; a++ )
    {
      p.pml_ad[a] = prof[0][a]; p.pml_bd[a] = prof[1][a]; p.pml_ah[a] = prof[2][a];
      p.pml_bh[a] = prof[3][a]; p.pml_ibd[a] = prof[4][a]; p.pml_ibh[a] = prof[5][a];
    }
  }
  vrefMurState( p.mur_flim , p.mur_zeta );

  /* Sources with their per-step amplitudes, as updateSourcesEfield/Hfield
   * compute them (src/source.c:600-753): size * wf(n dt) for E and
   * size * wf((n + 1/2) dt) for H; other source types act through the
   * coefficients set up at init. */
  int numSrc = vrefNumSources();
  vgpu_source *src = xcalloc( numSrc , sizeof( vgpu_source ) );
  double *srcValues = xcalloc( (size_t)numSrc * ( numSteps ? numSteps : 1 ) , sizeof( double ) );
  for( int q = 0 ; q < numSrc ; q++ )
  {
    int type , field , isSoft , flim[6];
    WaveformIndex wf;
    real size , delay;
    vrefSource( q , &type , &field , &isSoft , flim , &wf , &size , &delay );
    int kind;
    if( type == ST_EFIELD || type == ST_HFIELD )
      kind = VGPU_SRC_FIELD;
    else if( type == ST_ELEC_CURR_DENSITY || type == ST_MAGN_CURR_DENSITY )
      kind = VGPU_SRC_CURRENT;
    else
      continue;
    vgpu_source *o = &src[p.num_sources];
    double *v = srcValues + (size_t)p.num_sources * ( numSteps ? numSteps : 1 );
    o->field = field;
    o->kind = kind;
    o->soft = isSoft;
    for( int b = 0 ; b < 6 ; b++ ) o->flim[b] = flim[b];
    for( unsigned long n = 0 ; n < numSteps ; n++ )
    {
      real t = field <= EZ ? n * dt : ( n + 0.5 ) * dt;
      v[n] = size * getWaveformValue( t , wf , delay );
    }
    o->values = v;
    p.num_sources++;
  }
  p.sources = src;

  /* Every node an EH observer reads becomes a sampled point of the engine
   * (the low corner of an ASCII observer's box, every step-th node of a
   * binary observer's box); the reference's own observer code does the
   * rest. */
  int numObs = vrefNumObservers();
  size_t capacity = 0 , numPoints = 0;
  for( int pass = 0 ; pass < 2 ; pass++ )
  {
    for( int q = 0 ; q < numObs ; q++ )
    {
      int format , domain , quantity , gbbox[6] , step[3];
      vrefObserver( q , &format , &domain , &quantity , gbbox , step );
      if( quantity != OQ_EH ) continue;
      int hi[3] = { gbbox[XLO] , gbbox[YLO] , gbbox[ZLO] };
      if( format == OF_BINARY )
        for( int a = 0 ; a < 3 ; a++ ) hi[a] = gbbox[2 * a + 1];
      for( int k = gbbox[ZLO] ; k <= hi[2] ; k += format == OF_BINARY ? step[ZDIR] : 1 )
        for( int j = gbbox[YLO] ; j <= hi[1] ; j += format == OF_BINARY ? step[YDIR] : 1 )
          for( int i = gbbox[XLO] ; i <= hi[0] ; i += format == OF_BINARY ? step[XDIR] : 1 )
          {
            if( pass == 1 )
            {
              points[3 * numPoints] = i;
              points[3 * numPoints + 1] = j;
              points[3 * numPoints + 2] = k;
            }
            numPoints++;
          }
    }
    if( pass == 0 )
    {
      capacity = numPoints;
      numPoints = 0;
      points = xcalloc( 3 * capacity , sizeof( int ) );
    }
  }
  p.out_start = 0;
  p.out_stop = numSteps ? numSteps - 1 : 0;
  if( numPoints > 0x7fffffff / 6 )
    message( MSG_ERROR , 0 , "propagate (GPU): too many observer nodes\n" );
  p.num_td = (int)numPoints;
  p.td_points = points;

  message( MSG_LOG , 0 , "\nStarting time stepping loop on the GPU engine...\n" );
  startTimer( 0 , numSteps );
  check( vgpu_create( &p , &engine ) , "vgpu_create" );
  check( vgpu_run( engine , numSteps ) , "vgpu_run" );
  double *samples = xcalloc( (size_t)( numSteps ? numSteps : 1 ) * ( numPoints ? numPoints : 1 ) * 6 ,
                             sizeof( double ) );
  if( numPoints && numSteps )
    check( vgpu_read_td( engine , samples , numSteps ) , "vgpu_read_td" );
  vgpu_destroy( engine );

  /* The reference's observer pass of each step, on the engine's samples:
   * each node is set to the values it held at the top of that step. */
  real ***F[6] = { Ex , Ey , Ez , Hx , Hy , Hz };
  for( unsigned long n = 0 ; n < numSteps ; n++ )
  {
    for( size_t q = 0 ; q < numPoints ; q++ )
    {
      const double *s = samples + ( (size_t)n * numPoints + q ) * 6;
      int i = points[3 * q] , j = points[3 * q + 1] , k = points[3 * q + 2];
      for( int c = 0 ; c < 6 ; c++ ) F[c][i][j][k] = s[c];
    }
    real timeE = n * dt;
    updateObservers( n , timeE );
    updateWaveforms( n , timeE );
  }
  stopTimer( numSteps , numSteps );
  message( MSG_LOG , 0 , "\nCompleted time stepping loop.\n\n" );

  free( samples );
  free( points );
  free( srcValues );
  free( src );
}
