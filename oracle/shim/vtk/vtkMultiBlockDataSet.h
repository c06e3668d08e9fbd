// Stand-in header (oracle/_ref reference build only).
#include "vtk_shim.h"
