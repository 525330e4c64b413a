/* Scotch declarations for the single-rank oracle build.  With nParts = 1
 * every region gets one processor and mesh/mesh.cpp never reaches these
 * calls (mesh/mesh.cpp:784-792, 977-986); each stub aborts if it is. */
#ifndef HS_SHIM_SCOTCH_H
#define HS_SHIM_SCOTCH_H
typedef long SCOTCH_Num;
typedef struct { double opaque[16]; } SCOTCH_Graph;
typedef struct { double opaque[16]; } SCOTCH_Arch;
typedef struct { double opaque[16]; } SCOTCH_Strat;
#define SCOTCH_STRATQUALITY 1
int SCOTCH_graphInit(SCOTCH_Graph *);
int SCOTCH_graphBuild(SCOTCH_Graph *, SCOTCH_Num, SCOTCH_Num, const SCOTCH_Num *, const SCOTCH_Num *, const SCOTCH_Num *,
                      const SCOTCH_Num *, SCOTCH_Num, const SCOTCH_Num *, const SCOTCH_Num *);
int SCOTCH_archInit(SCOTCH_Arch *);
int SCOTCH_archCmplt(SCOTCH_Arch *, SCOTCH_Num);
int SCOTCH_stratInit(SCOTCH_Strat *);
int SCOTCH_stratGraphMapBuild(SCOTCH_Strat *, SCOTCH_Num, SCOTCH_Num, double);
int SCOTCH_graphMap(SCOTCH_Graph *, const SCOTCH_Arch *, SCOTCH_Strat *, SCOTCH_Num *);
#endif
