/* Oracle test infrastructure: marching-cubes tables (filled in with the mesh oracle). */
#include "mc_tables.h"
