// Space-group operation tables generated from International Tables (ITA Vol. A)
// generators, standard settings (monoclinic unique axis b, cell choice 1; origin
// choice 2 for the centrosymmetric groups that have two origins; hexagonal axes
// for rhombohedral groups).
//
// The reference obtains its operations from Crystalline.jl
// (`operations(spacegroup(sg, dim))`, src/symmetry_ops.jl:51-53), which is not
// available here.  This file replaces that dependency: every group is closed from
// its ITA generators in the order ITA lists general positions (coset
// representatives for the (0,0,0)+ set first, then one block per non-zero
// centering vector), and the fractional translations are converted to grid units
// exactly as `convert_op` does (src/symmetry_ops.jl:38-46).
#include "cfft_internal.h"

#include <cctype>
#include <cstring>
#include <string>
#include <vector>

namespace cfft {

namespace {

constexpr int DEN = 12;  // all ITA translations used here are multiples of 1/12

struct FracOp {
  int R[3][3];
  int t[3];  // numerators over DEN, reduced to [0, DEN)
};

struct GroupEntry {
  int sg;
  int dim;
  char centering;  // 'P','C','A','B','I','F','R' (3-D) ; 'p','c' (2-D)
  int order;       // expected number of operations including centering copies
  const char* gens;  // ';'-separated generators in ITA coordinate-triplet form
};

// Generators follow ITA's "generators selected" sequence (positions (2), (3), (5),
// (13), (25) ... of the general-position list).  `order` is |point group| times
// the number of centering translations.
const GroupEntry kGroups[] = {
    // ---------------- plane groups (dim = 2) ----------------
    {1, 2, 'p', 1, ""},
    {2, 2, 'p', 2, "-x,-y"},
    {3, 2, 'p', 2, "-x,y"},
    {4, 2, 'p', 2, "-x,y+1/2"},
    {5, 2, 'c', 4, "-x,y"},
    {6, 2, 'p', 4, "-x,-y;-x,y"},
    {7, 2, 'p', 4, "-x,-y;-x+1/2,y"},
    {8, 2, 'p', 4, "-x,-y;-x+1/2,y+1/2"},
    {9, 2, 'c', 8, "-x,-y;-x,y"},
    {10, 2, 'p', 4, "-x,-y;-y,x"},
    {11, 2, 'p', 8, "-x,-y;-y,x;-x,y"},
    {12, 2, 'p', 8, "-x,-y;-y,x;-x+1/2,y+1/2"},
    {13, 2, 'p', 3, "-y,x-y"},
    {14, 2, 'p', 6, "-y,x-y;-y,-x"},
    {15, 2, 'p', 6, "-y,x-y;y,x"},
    {16, 2, 'p', 6, "-y,x-y;-x,-y"},
    {17, 2, 'p', 12, "-y,x-y;-x,-y;-y,-x"},
    // ---------------- triclinic / monoclinic ----------------
    {1, 3, 'P', 1, ""},
    {2, 3, 'P', 2, "-x,-y,-z"},
    {3, 3, 'P', 2, "-x,y,-z"},
    {4, 3, 'P', 2, "-x,y+1/2,-z"},
    {5, 3, 'C', 4, "-x,y,-z"},
    {6, 3, 'P', 2, "x,-y,z"},
    {7, 3, 'P', 2, "x,-y,z+1/2"},
    {8, 3, 'C', 4, "x,-y,z"},
    {9, 3, 'C', 4, "x,-y,z+1/2"},
    {10, 3, 'P', 4, "-x,y,-z;-x,-y,-z"},
    {11, 3, 'P', 4, "-x,y+1/2,-z;-x,-y,-z"},
    {12, 3, 'C', 8, "-x,y,-z;-x,-y,-z"},
    {13, 3, 'P', 4, "-x,y,-z+1/2;-x,-y,-z"},
    {14, 3, 'P', 4, "-x,y+1/2,-z+1/2;-x,-y,-z"},
    {15, 3, 'C', 8, "-x,y,-z+1/2;-x,-y,-z"},
    // ---------------- orthorhombic ----------------
    {16, 3, 'P', 4, "-x,-y,z;-x,y,-z"},
    {17, 3, 'P', 4, "-x,-y,z+1/2;-x,y,-z+1/2"},
    {18, 3, 'P', 4, "-x,-y,z;-x+1/2,y+1/2,-z"},
    {19, 3, 'P', 4, "-x+1/2,-y,z+1/2;-x,y+1/2,-z+1/2"},
    {20, 3, 'C', 8, "-x,-y,z+1/2;-x,y,-z+1/2"},
    {21, 3, 'C', 8, "-x,-y,z;-x,y,-z"},
    {22, 3, 'F', 16, "-x,-y,z;-x,y,-z"},
    {23, 3, 'I', 8, "-x,-y,z;-x,y,-z"},
    {24, 3, 'I', 8, "-x+1/2,-y,z+1/2;-x,y+1/2,-z+1/2"},
    {25, 3, 'P', 4, "-x,-y,z;x,-y,z"},
    {26, 3, 'P', 4, "-x,-y,z+1/2;x,-y,z+1/2"},
    {27, 3, 'P', 4, "-x,-y,z;x,-y,z+1/2"},
    {28, 3, 'P', 4, "-x,-y,z;x+1/2,-y,z"},
    {29, 3, 'P', 4, "-x,-y,z+1/2;x+1/2,-y,z"},
    {30, 3, 'P', 4, "-x,-y,z;x,-y+1/2,z+1/2"},
    {31, 3, 'P', 4, "-x+1/2,-y,z+1/2;x+1/2,-y,z+1/2"},
    {32, 3, 'P', 4, "-x,-y,z;x+1/2,-y+1/2,z"},
    {33, 3, 'P', 4, "-x,-y,z+1/2;x+1/2,-y+1/2,z"},
    {34, 3, 'P', 4, "-x,-y,z;x+1/2,-y+1/2,z+1/2"},
    {35, 3, 'C', 8, "-x,-y,z;x,-y,z"},
    {36, 3, 'C', 8, "-x,-y,z+1/2;x,-y,z+1/2"},
    {37, 3, 'C', 8, "-x,-y,z;x,-y,z+1/2"},
    {38, 3, 'A', 8, "-x,-y,z;x,-y,z"},
    {39, 3, 'A', 8, "-x,-y,z;x,-y+1/2,z"},
    {40, 3, 'A', 8, "-x,-y,z;x+1/2,-y,z"},
    {41, 3, 'A', 8, "-x,-y,z;x+1/2,-y+1/2,z"},
    {42, 3, 'F', 16, "-x,-y,z;x,-y,z"},
    {43, 3, 'F', 16, "-x,-y,z;x+1/4,-y+1/4,z+1/4"},
    {44, 3, 'I', 8, "-x,-y,z;x,-y,z"},
    {45, 3, 'I', 8, "-x,-y,z;x+1/2,-y+1/2,z"},
    {46, 3, 'I', 8, "-x,-y,z;x+1/2,-y,z"},
    {47, 3, 'P', 8, "-x,-y,z;-x,y,-z;-x,-y,-z"},
    {48, 3, 'P', 8, "-x+1/2,-y+1/2,z;-x+1/2,y,-z+1/2;-x,-y,-z"},
    {49, 3, 'P', 8, "-x,-y,z;-x,y,-z+1/2;-x,-y,-z"},
    {50, 3, 'P', 8, "-x+1/2,-y+1/2,z;-x+1/2,y,-z;-x,-y,-z"},
    {51, 3, 'P', 8, "-x+1/2,-y,z;-x,y,-z;-x,-y,-z"},
    {52, 3, 'P', 8, "-x+1/2,-y,z;-x+1/2,y+1/2,-z+1/2;-x,-y,-z"},
    {53, 3, 'P', 8, "-x+1/2,-y,z+1/2;-x+1/2,y,-z+1/2;-x,-y,-z"},
    {54, 3, 'P', 8, "-x+1/2,-y,z;-x,y,-z+1/2;-x,-y,-z"},
    {55, 3, 'P', 8, "-x,-y,z;-x+1/2,y+1/2,-z;-x,-y,-z"},
    {56, 3, 'P', 8, "-x+1/2,-y+1/2,z;-x,y+1/2,-z+1/2;-x,-y,-z"},
    {57, 3, 'P', 8, "-x,-y,z+1/2;-x,y+1/2,-z+1/2;-x,-y,-z"},
    {58, 3, 'P', 8, "-x,-y,z;-x+1/2,y+1/2,-z+1/2;-x,-y,-z"},
    {59, 3, 'P', 8, "-x+1/2,-y+1/2,z;-x,y+1/2,-z;-x,-y,-z"},
    {60, 3, 'P', 8, "-x+1/2,-y+1/2,z+1/2;-x,y,-z+1/2;-x,-y,-z"},
    {61, 3, 'P', 8, "-x+1/2,-y,z+1/2;-x,y+1/2,-z+1/2;-x,-y,-z"},
    {62, 3, 'P', 8, "-x+1/2,-y,z+1/2;-x,y+1/2,-z;-x,-y,-z"},
    {63, 3, 'C', 16, "-x,-y,z+1/2;-x,y,-z+1/2;-x,-y,-z"},
    {64, 3, 'C', 16, "-x,-y+1/2,z+1/2;-x,y+1/2,-z+1/2;-x,-y,-z"},
    {65, 3, 'C', 16, "-x,-y,z;-x,y,-z;-x,-y,-z"},
    {66, 3, 'C', 16, "-x,-y,z;-x,y,-z+1/2;-x,-y,-z"},
    {67, 3, 'C', 16, "-x,-y+1/2,z;-x,y+1/2,-z;-x,-y,-z"},
    {68, 3, 'C', 16, "-x+1/2,-y,z;-x,y,-z+1/2;-x,-y,-z"},
    {69, 3, 'F', 32, "-x,-y,z;-x,y,-z;-x,-y,-z"},
    {70, 3, 'F', 32, "-x+3/4,-y+3/4,z;-x+3/4,y,-z+3/4;-x,-y,-z"},
    {71, 3, 'I', 16, "-x,-y,z;-x,y,-z;-x,-y,-z"},
    {72, 3, 'I', 16, "-x,-y,z;-x+1/2,y+1/2,-z;-x,-y,-z"},
    {73, 3, 'I', 16, "-x+1/2,-y,z+1/2;-x,y+1/2,-z+1/2;-x,-y,-z"},
    {74, 3, 'I', 16, "-x,-y+1/2,z;-x,y+1/2,-z;-x,-y,-z"},
    // ---------------- tetragonal (all 68; origin choice 2 where there are two) ----------------
    {75, 3, 'P', 4, "-x,-y,z;-y,x,z"},
    {76, 3, 'P', 4, "-x,-y,z+1/2;-y,x,z+1/4"},
    {77, 3, 'P', 4, "-x,-y,z;-y,x,z+1/2"},
    {78, 3, 'P', 4, "-x,-y,z+1/2;-y,x,z+3/4"},
    {79, 3, 'I', 8, "-x,-y,z;-y,x,z"},
    {80, 3, 'I', 8, "-x+1/2,-y+1/2,z+1/2;-y,x+1/2,z+1/4"},
    {81, 3, 'P', 4, "-x,-y,z;y,-x,-z"},
    {82, 3, 'I', 8, "-x,-y,z;y,-x,-z"},
    {83, 3, 'P', 8, "-x,-y,z;-y,x,z;-x,-y,-z"},
    {84, 3, 'P', 8, "-x,-y,z;-y,x,z+1/2;-x,-y,-z"},
    {85, 3, 'P', 8, "-x+1/2,-y+1/2,z;-y+1/2,x,z;-x,-y,-z"},
    {86, 3, 'P', 8, "-x+1/2,-y+1/2,z;-y,x+1/2,z+1/2;-x,-y,-z"},
    {87, 3, 'I', 16, "-x,-y,z;-y,x,z;-x,-y,-z"},
    {88, 3, 'I', 16, "-x+1/2,-y,z+1/2;-y+3/4,x+1/4,z+1/4;-x,-y,-z"},
    {89, 3, 'P', 8, "-x,-y,z;-y,x,z;-x,y,-z"},
    {90, 3, 'P', 8, "-x,-y,z;-y+1/2,x+1/2,z;-x+1/2,y+1/2,-z"},
    {91, 3, 'P', 8, "-x,-y,z+1/2;-y,x,z+1/4;-x,y,-z"},
    {92, 3, 'P', 8, "-x,-y,z+1/2;-y+1/2,x+1/2,z+1/4;-x+1/2,y+1/2,-z+1/4"},
    {93, 3, 'P', 8, "-x,-y,z;-y,x,z+1/2;-x,y,-z"},
    {94, 3, 'P', 8, "-x,-y,z;-y+1/2,x+1/2,z+1/2;-x+1/2,y+1/2,-z+1/2"},
    {95, 3, 'P', 8, "-x,-y,z+1/2;-y,x,z+3/4;-x,y,-z"},
    {96, 3, 'P', 8, "-x,-y,z+1/2;-y+1/2,x+1/2,z+3/4;-x+1/2,y+1/2,-z+3/4"},
    {97, 3, 'I', 16, "-x,-y,z;-y,x,z;-x,y,-z"},
    {98, 3, 'I', 16, "-x+1/2,-y+1/2,z+1/2;-y,x+1/2,z+1/4;-x+1/2,y,-z+3/4"},
    {99, 3, 'P', 8, "-x,-y,z;-y,x,z;x,-y,z"},
    {100, 3, 'P', 8, "-x,-y,z;-y,x,z;x+1/2,-y+1/2,z"},
    {101, 3, 'P', 8, "-x,-y,z;-y,x,z+1/2;x,-y,z+1/2"},
    {102, 3, 'P', 8, "-x,-y,z;-y+1/2,x+1/2,z+1/2;x+1/2,-y+1/2,z+1/2"},
    {103, 3, 'P', 8, "-x,-y,z;-y,x,z;x,-y,z+1/2"},
    {104, 3, 'P', 8, "-x,-y,z;-y,x,z;x+1/2,-y+1/2,z+1/2"},
    {105, 3, 'P', 8, "-x,-y,z;-y,x,z+1/2;x,-y,z"},
    {106, 3, 'P', 8, "-x,-y,z;-y,x,z+1/2;x+1/2,-y+1/2,z"},
    {107, 3, 'I', 16, "-x,-y,z;-y,x,z;x,-y,z"},
    {108, 3, 'I', 16, "-x,-y,z;-y,x,z;x,-y,z+1/2"},
    {109, 3, 'I', 16, "-x+1/2,-y+1/2,z+1/2;-y,x+1/2,z+1/4;x,-y,z"},
    {110, 3, 'I', 16, "-x+1/2,-y+1/2,z+1/2;-y,x+1/2,z+1/4;x,-y,z+1/2"},
    {111, 3, 'P', 8, "-x,-y,z;y,-x,-z;-x,y,-z"},
    {112, 3, 'P', 8, "-x,-y,z;y,-x,-z;-x,y,-z+1/2"},
    {113, 3, 'P', 8, "-x,-y,z;y,-x,-z;-x+1/2,y+1/2,-z"},
    {114, 3, 'P', 8, "-x,-y,z;y,-x,-z;-x+1/2,y+1/2,-z+1/2"},
    {115, 3, 'P', 8, "-x,-y,z;y,-x,-z;x,-y,z"},
    {116, 3, 'P', 8, "-x,-y,z;y,-x,-z;x,-y,z+1/2"},
    {117, 3, 'P', 8, "-x,-y,z;y,-x,-z;x+1/2,-y+1/2,z"},
    {118, 3, 'P', 8, "-x,-y,z;y,-x,-z;x+1/2,-y+1/2,z+1/2"},
    {119, 3, 'I', 16, "-x,-y,z;y,-x,-z;x,-y,z"},
    {120, 3, 'I', 16, "-x,-y,z;y,-x,-z;x,-y,z+1/2"},
    {121, 3, 'I', 16, "-x,-y,z;y,-x,-z;-x,y,-z"},
    {122, 3, 'I', 16, "-x,-y,z;y,-x,-z;-x+1/2,y,-z+3/4"},
    {123, 3, 'P', 16, "-x,-y,z;-y,x,z;-x,y,-z;-x,-y,-z"},
    {124, 3, 'P', 16, "-x,-y,z;-y,x,z;-x,y,-z+1/2;-x,-y,-z"},
    {125, 3, 'P', 16, "-x+1/2,-y+1/2,z;-y+1/2,x,z;-x+1/2,y,-z;-x,-y,-z"},
    {126, 3, 'P', 16, "-x+1/2,-y+1/2,z;-y+1/2,x,z;-x+1/2,y,-z+1/2;-x,-y,-z"},
    {127, 3, 'P', 16, "-x,-y,z;-y,x,z;-x+1/2,y+1/2,-z;-x,-y,-z"},
    {128, 3, 'P', 16, "-x,-y,z;-y,x,z;-x+1/2,y+1/2,-z+1/2;-x,-y,-z"},
    {129, 3, 'P', 16, "-x+1/2,-y+1/2,z;-y+1/2,x,z;-x,y+1/2,-z;-x,-y,-z"},
    {130, 3, 'P', 16, "-x+1/2,-y+1/2,z;-y+1/2,x,z;-x,y+1/2,-z+1/2;-x,-y,-z"},
    {131, 3, 'P', 16, "-x,-y,z;-y,x,z+1/2;-x,y,-z;-x,-y,-z"},
    {132, 3, 'P', 16, "-x,-y,z;-y,x,z+1/2;-x,y,-z+1/2;-x,-y,-z"},
    {133, 3, 'P', 16, "-x+1/2,-y+1/2,z;-y+1/2,x,z+1/2;-x+1/2,y,-z;-x,-y,-z"},
    {134, 3, 'P', 16, "-x+1/2,-y+1/2,z;-y+1/2,x,z+1/2;-x+1/2,y,-z+1/2;-x,-y,-z"},
    {135, 3, 'P', 16, "-x,-y,z;-y,x,z+1/2;-x+1/2,y+1/2,-z;-x,-y,-z"},
    {136, 3, 'P', 16, "-x,-y,z;-y+1/2,x+1/2,z+1/2;-x+1/2,y+1/2,-z+1/2;-x,-y,-z"},
    {137, 3, 'P', 16, "-x+1/2,-y+1/2,z;-y+1/2,x,z+1/2;-x,y+1/2,-z;-x,-y,-z"},
    {138, 3, 'P', 16, "-x+1/2,-y+1/2,z;-y+1/2,x,z+1/2;-x,y+1/2,-z+1/2;-x,-y,-z"},
    {139, 3, 'I', 32, "-x,-y,z;-y,x,z;-x,y,-z;-x,-y,-z"},
    {140, 3, 'I', 32, "-x,-y,z;-y,x,z;-x,y,-z+1/2;-x,-y,-z"},
    {141, 3, 'I', 32, "-x+1/2,-y,z+1/2;-y+1/4,x+3/4,z+1/4;-x+1/2,y,-z+1/2;-x,-y,-z"},
    {142, 3, 'I', 32, "-x+1/2,-y,z+1/2;-y+1/4,x+3/4,z+1/4;-x+1/2,y,-z;-x,-y,-z"},
    // ---------------- trigonal / hexagonal (all 52, hexagonal axes; R obverse) ----------
    {143, 3, 'P', 3, "-y,x-y,z"},
    {144, 3, 'P', 3, "-y,x-y,z+1/3"},
    {145, 3, 'P', 3, "-y,x-y,z+2/3"},
    {146, 3, 'R', 9, "-y,x-y,z"},
    {147, 3, 'P', 6, "-y,x-y,z;-x,-y,-z"},
    {148, 3, 'R', 18, "-y,x-y,z;-x,-y,-z"},
    {149, 3, 'P', 6, "-y,x-y,z;-y,-x,-z"},
    {150, 3, 'P', 6, "-y,x-y,z;y,x,-z"},
    {151, 3, 'P', 6, "-y,x-y,z+1/3;-y,-x,-z+2/3"},
    {152, 3, 'P', 6, "-y,x-y,z+1/3;y,x,-z"},
    {153, 3, 'P', 6, "-y,x-y,z+2/3;-y,-x,-z+1/3"},
    {154, 3, 'P', 6, "-y,x-y,z+2/3;y,x,-z"},
    {155, 3, 'R', 18, "-y,x-y,z;y,x,-z"},
    {156, 3, 'P', 6, "-y,x-y,z;-y,-x,z"},
    {157, 3, 'P', 6, "-y,x-y,z;y,x,z"},
    {158, 3, 'P', 6, "-y,x-y,z;-y,-x,z+1/2"},
    {159, 3, 'P', 6, "-y,x-y,z;y,x,z+1/2"},
    {160, 3, 'R', 18, "-y,x-y,z;-y,-x,z"},
    {161, 3, 'R', 18, "-y,x-y,z;-y,-x,z+1/2"},
    {162, 3, 'P', 12, "-y,x-y,z;-y,-x,-z;-x,-y,-z"},
    {163, 3, 'P', 12, "-y,x-y,z;-y,-x,-z+1/2;-x,-y,-z"},
    {164, 3, 'P', 12, "-y,x-y,z;y,x,-z;-x,-y,-z"},
    {165, 3, 'P', 12, "-y,x-y,z;y,x,-z+1/2;-x,-y,-z"},
    {166, 3, 'R', 36, "-y,x-y,z;y,x,-z;-x,-y,-z"},
    {167, 3, 'R', 36, "-y,x-y,z;y,x,-z+1/2;-x,-y,-z"},
    {168, 3, 'P', 6, "-y,x-y,z;-x,-y,z"},
    {169, 3, 'P', 6, "-y,x-y,z+1/3;-x,-y,z+1/2"},
    {170, 3, 'P', 6, "-y,x-y,z+2/3;-x,-y,z+1/2"},
    {171, 3, 'P', 6, "-y,x-y,z+2/3;-x,-y,z"},
    {172, 3, 'P', 6, "-y,x-y,z+1/3;-x,-y,z"},
    {173, 3, 'P', 6, "-y,x-y,z;-x,-y,z+1/2"},
    {174, 3, 'P', 6, "-y,x-y,z;x,y,-z"},
    {175, 3, 'P', 12, "-y,x-y,z;-x,-y,z;-x,-y,-z"},
    {176, 3, 'P', 12, "-y,x-y,z;-x,-y,z+1/2;-x,-y,-z"},
    {177, 3, 'P', 12, "-y,x-y,z;-x,-y,z;y,x,-z"},
    {178, 3, 'P', 12, "-y,x-y,z+1/3;-x,-y,z+1/2;y,x,-z+1/3"},
    {179, 3, 'P', 12, "-y,x-y,z+2/3;-x,-y,z+1/2;y,x,-z+2/3"},
    {180, 3, 'P', 12, "-y,x-y,z+2/3;-x,-y,z;y,x,-z+2/3"},
    {181, 3, 'P', 12, "-y,x-y,z+1/3;-x,-y,z;y,x,-z+1/3"},
    {182, 3, 'P', 12, "-y,x-y,z;-x,-y,z+1/2;y,x,-z"},
    {183, 3, 'P', 12, "-y,x-y,z;-x,-y,z;-y,-x,z"},
    {184, 3, 'P', 12, "-y,x-y,z;-x,-y,z;-y,-x,z+1/2"},
    {185, 3, 'P', 12, "-y,x-y,z;-x,-y,z+1/2;-y,-x,z+1/2"},
    {186, 3, 'P', 12, "-y,x-y,z;-x,-y,z+1/2;-y,-x,z"},
    {187, 3, 'P', 12, "-y,x-y,z;x,y,-z;-y,-x,z"},
    {188, 3, 'P', 12, "-y,x-y,z;x,y,-z+1/2;-y,-x,z+1/2"},
    {189, 3, 'P', 12, "-y,x-y,z;x,y,-z;y,x,-z"},
    {190, 3, 'P', 12, "-y,x-y,z;x,y,-z+1/2;y,x,-z"},
    {191, 3, 'P', 24, "-y,x-y,z;-x,-y,z;y,x,-z;-x,-y,-z"},
    {192, 3, 'P', 24, "-y,x-y,z;-x,-y,z;y,x,-z+1/2;-x,-y,-z"},
    {193, 3, 'P', 24, "-y,x-y,z;-x,-y,z+1/2;y,x,-z+1/2;-x,-y,-z"},
    {194, 3, 'P', 24, "-y,x-y,z;-x,-y,z+1/2;y,x,-z;-x,-y,-z"},
    // ---------------- cubic (all 36) ----------------
    {195, 3, 'P', 12, "-x,-y,z;-x,y,-z;z,x,y"},
    {196, 3, 'F', 48, "-x,-y,z;-x,y,-z;z,x,y"},
    {197, 3, 'I', 24, "-x,-y,z;-x,y,-z;z,x,y"},
    {198, 3, 'P', 12, "-x+1/2,-y,z+1/2;-x,y+1/2,-z+1/2;z,x,y"},
    {199, 3, 'I', 24, "-x+1/2,-y,z+1/2;-x,y+1/2,-z+1/2;z,x,y"},
    {200, 3, 'P', 24, "-x,-y,z;-x,y,-z;z,x,y;-x,-y,-z"},
    {201, 3, 'P', 24, "-x+1/2,-y+1/2,z;-x+1/2,y,-z+1/2;z,x,y;-x,-y,-z"},
    {202, 3, 'F', 96, "-x,-y,z;-x,y,-z;z,x,y;-x,-y,-z"},
    {203, 3, 'F', 96, "-x+3/4,-y+3/4,z;-x+3/4,y,-z+3/4;z,x,y;-x,-y,-z"},
    {204, 3, 'I', 48, "-x,-y,z;-x,y,-z;z,x,y;-x,-y,-z"},
    {205, 3, 'P', 24, "-x+1/2,-y,z+1/2;-x,y+1/2,-z+1/2;z,x,y;-x,-y,-z"},
    {206, 3, 'I', 48, "-x+1/2,-y,z+1/2;-x,y+1/2,-z+1/2;z,x,y;-x,-y,-z"},
    {207, 3, 'P', 24, "-x,-y,z;-x,y,-z;z,x,y;y,x,-z"},
    {208, 3, 'P', 24, "-x,-y,z;-x,y,-z;z,x,y;y+1/2,x+1/2,-z+1/2"},
    {209, 3, 'F', 96, "-x,-y,z;-x,y,-z;z,x,y;y,x,-z"},
    {210, 3, 'F', 96, "-x,-y+1/2,z+1/2;-x+1/2,y+1/2,-z;z,x,y;y+3/4,x+1/4,-z+3/4"},
    {211, 3, 'I', 48, "-x,-y,z;-x,y,-z;z,x,y;y,x,-z"},
    {212, 3, 'P', 24, "-x+1/2,-y,z+1/2;-x,y+1/2,-z+1/2;z,x,y;y+1/4,x+3/4,-z+3/4"},
    {213, 3, 'P', 24, "-x+1/2,-y,z+1/2;-x,y+1/2,-z+1/2;z,x,y;y+3/4,x+1/4,-z+1/4"},
    {214, 3, 'I', 48, "-x+1/2,-y,z+1/2;-x,y+1/2,-z+1/2;z,x,y;y+3/4,x+1/4,-z+1/4"},
    {215, 3, 'P', 24, "-x,-y,z;-x,y,-z;z,x,y;y,x,z"},
    {216, 3, 'F', 96, "-x,-y,z;-x,y,-z;z,x,y;y,x,z"},
    {217, 3, 'I', 48, "-x,-y,z;-x,y,-z;z,x,y;y,x,z"},
    {218, 3, 'P', 24, "-x,-y,z;-x,y,-z;z,x,y;y+1/2,x+1/2,z+1/2"},
    {219, 3, 'F', 96, "-x,-y,z;-x,y,-z;z,x,y;y+1/2,x+1/2,z+1/2"},
    {220, 3, 'I', 48, "-x+1/2,-y,z+1/2;-x,y+1/2,-z+1/2;z,x,y;y+1/4,x+1/4,z+1/4"},
    {221, 3, 'P', 48, "-x,-y,z;-x,y,-z;z,x,y;y,x,-z;-x,-y,-z"},
    {222, 3, 'P', 48, "-x+1/2,-y+1/2,z;-x+1/2,y,-z+1/2;z,x,y;y,x,-z+1/2;-x,-y,-z"},
    {223, 3, 'P', 48, "-x,-y,z;-x,y,-z;z,x,y;y+1/2,x+1/2,-z+1/2;-x,-y,-z"},
    {224, 3, 'P', 48, "-x+1/2,-y+1/2,z;-x+1/2,y,-z+1/2;z,x,y;y+1/2,x+1/2,-z;-x,-y,-z"},
    {225, 3, 'F', 192, "-x,-y,z;-x,y,-z;z,x,y;y,x,-z;-x,-y,-z"},
    {226, 3, 'F', 192, "-x,-y,z;-x,y,-z;z,x,y;y+1/2,x+1/2,-z+1/2;-x,-y,-z"},
    {227, 3, 'F', 192, "-x+3/4,-y+1/4,z+1/2;-x+1/4,y+1/2,-z+3/4;z,x,y;y+3/4,x+1/4,-z+1/2;-x,-y,-z"},
    {228, 3, 'F', 192, "-x+1/4,-y+3/4,z+1/2;-x+3/4,y+1/2,-z+1/4;z,x,y;y+3/4,x+1/4,-z;-x,-y,-z"},
    {229, 3, 'I', 96, "-x,-y,z;-x,y,-z;z,x,y;y,x,-z;-x,-y,-z"},
    {230, 3, 'I', 96, "-x+1/2,-y,z+1/2;-x,y+1/2,-z+1/2;z,x,y;y+3/4,x+1/4,-z+1/4;-x,-y,-z"},
};

int mod_den(int v) {
  int r = v % DEN;
  return r < 0 ? r + DEN : r;
}

FracOp identity_op() {
  FracOp op{};
  for (int i = 0; i < 3; ++i) op.R[i][i] = 1;
  return op;
}

// Parse one ITA coordinate triplet such as "-x+y,x-1/4,-z+3/4" (2 or 3 terms).
bool parse_triplet(const std::string& s, int dim, FracOp* out, std::string* err) {
  FracOp op{};
  int comp = 0;
  size_t i = 0;
  while (comp < dim) {
    int sign = 1;
    bool any = false;
    while (i < s.size() && s[i] != ',') {
      char c = s[i];
      if (c == ' ') { ++i; continue; }
      if (c == '+') { sign = 1; ++i; continue; }
      if (c == '-') { sign = -1; ++i; continue; }
      if (c == 'x' || c == 'y' || c == 'z') {
        int ax = c - 'x';
        if (ax >= dim) { *err = "axis beyond dimension in '" + s + "'"; return false; }
        op.R[comp][ax] += sign;
        sign = 1; any = true; ++i;
        continue;
      }
      if (std::isdigit(static_cast<unsigned char>(c))) {
        int num = 0;
        while (i < s.size() && std::isdigit(static_cast<unsigned char>(s[i]))) num = num * 10 + (s[i++] - '0');
        int den = 1;
        if (i < s.size() && s[i] == '/') {
          ++i; den = 0;
          while (i < s.size() && std::isdigit(static_cast<unsigned char>(s[i]))) den = den * 10 + (s[i++] - '0');
        }
        if (den <= 0 || (num * DEN) % den != 0) { *err = "translation not a multiple of 1/12 in '" + s + "'"; return false; }
        op.t[comp] += sign * num * DEN / den;
        sign = 1; any = true;
        continue;
      }
      *err = std::string("unexpected character in '") + s + "'";
      return false;
    }
    if (!any) { *err = "empty component in '" + s + "'"; return false; }
    op.t[comp] = mod_den(op.t[comp]);
    ++comp;
    if (i < s.size() && s[i] == ',') ++i;
  }
  for (int d = dim; d < 3; ++d) op.R[d][d] = 1;
  *out = op;
  return true;
}

// a ∘ b : x -> Ra (Rb x + tb) + ta
FracOp compose(const FracOp& a, const FracOp& b) {
  FracOp c{};
  for (int i = 0; i < 3; ++i) {
    int tt = a.t[i];
    for (int j = 0; j < 3; ++j) {
      int s = 0;
      for (int k = 0; k < 3; ++k) s += a.R[i][k] * b.R[k][j];
      c.R[i][j] = s;
      tt += a.R[i][j] * b.t[j];
    }
    c.t[i] = mod_den(tt);
  }
  return c;
}

bool same_R(const FracOp& a, const FracOp& b) {
  return std::memcmp(a.R, b.R, sizeof(a.R)) == 0;
}

std::vector<std::array<int, 3>> centering_vectors(char c, int dim) {
  std::vector<std::array<int, 3>> v;
  const int h = DEN / 2;
  switch (c) {
    case 'C': v.push_back({h, h, 0}); break;
    case 'A': v.push_back({0, h, h}); break;
    case 'B': v.push_back({h, 0, h}); break;
    case 'I': v.push_back({h, h, h}); break;
    case 'F': v.push_back({0, h, h}); v.push_back({h, 0, h}); v.push_back({h, h, 0}); break;
    case 'R': v.push_back({8, 4, 4}); v.push_back({4, 8, 8}); break;
    case 'c': v.push_back({h, h, 0}); break;
    default: break;
  }
  (void)dim;
  return v;
}

// Equality modulo the (centred) lattice.
bool equal_mod_lattice(const FracOp& a, const FracOp& b, const std::vector<std::array<int, 3>>& cvec) {
  if (!same_R(a, b)) return false;
  int d[3];
  for (int i = 0; i < 3; ++i) d[i] = mod_den(a.t[i] - b.t[i]);
  if (d[0] == 0 && d[1] == 0 && d[2] == 0) return true;
  for (const auto& c : cvec)
    if (d[0] == c[0] && d[1] == c[1] && d[2] == c[2]) return true;
  return false;
}

bool contains(const std::vector<FracOp>& H, const FracOp& g, const std::vector<std::array<int, 3>>& cvec) {
  for (const auto& h : H)
    if (equal_mod_lattice(h, g, cvec)) return true;
  return false;
}

const GroupEntry* find_entry(int sg, int dim) {
  for (const auto& e : kGroups)
    if (e.sg == sg && e.dim == dim) return &e;
  return nullptr;
}

}  // namespace

bool has_group(int sg, int dim) { return find_entry(sg, dim) != nullptr; }

int list_groups(int dim, int* out, int cap) {
  int n = 0;
  for (const auto& e : kGroups)
    if (e.dim == dim) {
      if (out && n < cap) out[n] = e.sg;
      ++n;
    }
  return n;
}

// Fractional ops (translations in 1/12) in ITA listing order.
static bool generate_fractional(int sg, int dim, std::vector<FracOp>* ops, std::string* err) {
  const GroupEntry* e = find_entry(sg, dim);
  if (!e) { *err = "space group " + std::to_string(sg) + " (dim " + std::to_string(dim) + ") is not in the built-in table"; return false; }
  std::vector<FracOp> gens;
  std::string g = e->gens;
  size_t pos = 0;
  while (pos < g.size()) {
    size_t nxt = g.find(';', pos);
    if (nxt == std::string::npos) nxt = g.size();
    FracOp op;
    if (!parse_triplet(g.substr(pos, nxt - pos), dim, &op, err)) return false;
    gens.push_back(op);
    pos = nxt + 1;
  }
  const auto cvec = centering_vectors(e->centering, dim);
  std::vector<FracOp> H{identity_op()};
  for (const auto& gen : gens) {
    if (contains(H, gen, cvec)) continue;
    const std::vector<FracOp> base = H;
    FracOp gk = gen;
    int guard = 0;
    while (!contains(base, gk, cvec)) {
      for (const auto& h : base) H.push_back(compose(gk, h));
      gk = compose(gen, gk);
      if (++guard > 12) { *err = "generator power did not return to the subgroup"; return false; }
    }
  }
  // Verify closure modulo the centred lattice.
  for (const auto& a : H)
    for (const auto& b : H)
      if (!contains(H, compose(a, b), cvec)) { *err = "generated set is not closed for group " + std::to_string(sg); return false; }
  std::vector<FracOp> full = H;
  for (const auto& c : cvec)
    for (const auto& h : H) {
      FracOp o = h;
      for (int i = 0; i < 3; ++i) o.t[i] = mod_den(o.t[i] + c[i]);
      full.push_back(o);
    }
  if (static_cast<int>(full.size()) != e->order) {
    *err = "group " + std::to_string(sg) + " closed to " + std::to_string(full.size()) + " operations, expected " + std::to_string(e->order);
    return false;
  }
  *ops = full;
  return true;
}

Status get_ops(int sg, int dim, const int* N, std::vector<SymOp>* out, std::string* err) {
  if (dim != 2 && dim != 3) { *err = "dim must be 2 or 3"; return Status::kInvalid; }
  std::vector<FracOp> frac;
  if (!generate_fractional(sg, dim, &frac, err)) return Status::kUnsupported;
  out->clear();
  for (const auto& f : frac) {
    SymOp op{};
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) op.R[i][j] = f.R[i][j];
    for (int d = 0; d < 3; ++d) {
      const int n = d < dim ? N[d] : 1;
      if (d >= dim) { op.t[d] = 0; continue; }
      // convert_op: t_grid = t_frac * N must be an integer (src/symmetry_ops.jl:38-46)
      const long num = static_cast<long>(f.t[d]) * n;
      if (num % DEN != 0) {
        *err = "Symmetry operation not commensurate with grid";
        return Status::kNotCommensurate;
      }
      op.t[d] = static_cast<int>(num / DEN);
    }
    out->push_back(op);
  }
  return Status::kOk;
}

}  // namespace cfft
