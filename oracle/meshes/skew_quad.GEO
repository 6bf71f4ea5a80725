skewed quadrilateral, not a parallelogram; vertices by (component, parameter)
Parametrisierung PARXC PARYC TMAXC
      1   4   0   4     1       NEL NVT NMT NVE NBCT
DCORVG
   0   0
   1   0
   2   0
   3   0
KVERT
   1  2  3  4
KNPR
  1  1  1  1
KMM
1 4
