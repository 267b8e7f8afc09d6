
/* ---- appended by oracle/build_ref.sh to a copy of source.c ----
 * The source list in its update order, for the propagate() replacement of
 * oracle/propagate_gpu/propagate_gpu.c. */
int vrefNumSources( void )
{
  int n = 0;
  SourceItem *item;
  DL_FOREACH( sourceList , item ) n++;
  return n;
}

void vrefSource( int q , int *type , int *field , int *isSoft , int flim[6] , WaveformIndex *waveform ,
                 real *size , real *delay )
{
  int n = 0;
  SourceItem *item;
  DL_FOREACH( sourceList , item )
  {
    if( n++ != q ) continue;
    *type = item->type;
    *field = item->field;
    *isSoft = item->isSoft;
    for( int b = 0 ; b < 6 ; b++ ) flim[b] = item->flim[item->field][b];
    *waveform = item->waveformNumber;
    *size = item->size;
    *delay = item->delay;
  }
}
