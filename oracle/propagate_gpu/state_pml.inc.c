
/* ---- appended by oracle/build_ref.sh to a copy of pml.c ----
 * The UPML module's private state for the propagate() replacement of
 * oracle/propagate_gpu/propagate_gpu.c: which regions the update loops visit
 * (those with auxiliary arrays, updatePmlEfield's own test at pml.c:884),
 * their field limits and the loss-profile lines of each axis. */
void vrefPmlState( int present[6] , int lim[6][6][6] , real *prof[6][3] )
{
  real *p[6][3] = { { adx , ady , adz } , { bdx , bdy , bdz } , { ahx , ahy , ahz } ,
                    { bhx , bhy , bhz } , { ibdx , ibdy , ibdz } , { ibhx , ibhy , ibhz } };
  for( int r = 0 ; r < 6 ; r++ )
    present[r] = Px[r] != NULL;
  for( int r = 0 ; r < 6 ; r++ )
    for( int f = 0 ; f < 6 ; f++ )
      for( int b = 0 ; b < 6 ; b++ )
        lim[r][f][b] = fplim[r][f][b];
  for( int q = 0 ; q < 6 ; q++ )
    for( int a = 0 ; a < 3 ; a++ )
      prof[q][a] = p[q][a];
}
