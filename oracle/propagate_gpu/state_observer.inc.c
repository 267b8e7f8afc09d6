
/* ---- appended by oracle/build_ref.sh to a copy of observer.c ----
 * The observer list, for the propagate() replacement of
 * oracle/propagate_gpu/propagate_gpu.c: each observer's format, domain,
 * quantity, grid bounding box and node steps (an ASCII EH observer samples
 * the six components at its box's low corner, observer.c:776-778; a binary
 * one every step-th node of its box, observer.c:1171-1173). */
int vrefNumObservers( void )
{
  int n = 0;
  ObserverItem *item;
  DL_FOREACH( observerList , item ) n++;
  return n;
}

void vrefObserver( int q , int *format , int *domain , int *quantity , int gbbox[6] , int step[3] )
{
  int n = 0;
  ObserverItem *item;
  DL_FOREACH( observerList , item )
  {
    if( n++ != q ) continue;
    *format = item->format;
    *domain = item->domain;
    *quantity = item->quantity;
    for( int b = 0 ; b < 6 ; b++ ) gbbox[b] = item->gbbox[b];
    for( int a = 0 ; a < 3 ; a++ ) step[a] = item->step[a];
  }
}
