
/* ---- appended by oracle/build_ref.sh to a copy of mur.c ----
 * First-order Mur faces' field limits and phase factors, for the
 * propagate() replacement of oracle/propagate_gpu/propagate_gpu.c. */
void vrefMurState( int lim[6][6][6] , real z[6] )
{
  for( int r = 0 ; r < 6 ; r++ )
  {
    z[r] = zeta[r];
    for( int f = 0 ; f < 6 ; f++ )
      for( int b = 0 ; b < 6 ; b++ )
        lim[r][f][b] = fmlim[r][f][b];
  }
}
