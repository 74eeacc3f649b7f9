/* shim: see mdb.h */
#include "mdb.h"
