/* Stands in for the reference header of the same name: a reference driver compiled with
 * this directory ahead of the reference's own on its include path gets swift_compat.h (the
 * library's functions under the reference's names) wherever it includes balance.h. */
#include "swift_compat.h"
