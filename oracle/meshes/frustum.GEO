pyramid frustum, not a parallelepiped; explicit coordinates (KNPR 0)
Parametrisierung
       1    8    4    8    6         NEL NVT NVpF NVpEL NBF
DCORVG (comp, t, s  or  x, y, z)
 0 0 0
 1 0 0
 1 1 0
 0 1 0
 0.14000000000000001 0.080000000000000002 1
 0.94000000000000006 0.080000000000000002 1
 0.94000000000000006 0.88 1
 0.14000000000000001 0.88 1
KVERT
   1   2   3   4   5   6   7   8
KNPR
   0   0   0   0   0   0   0   0
BoundFaces
   1   2   3   4
   1   2   6   5
   2   3   7   6
   3   4   8   7
   4   1   5   8
   5   6   7   8
FaceParam (cell, locface, boundary part/component)
   1   1   1   1
   1   2   1   3
   1   3   1   5
   1   4   1   6
   1   5   1   2
   1   6   1   4
