/* Stand-in header: the classes are in ref_context.h (test infrastructure). */
#include "ref_context.h"
