/* shim: everything lives in HYPRE.h */
#include "HYPRE.h"
