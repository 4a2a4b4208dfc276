// Where the reference's sources include <ampcor/correlators.h> (the installed name of
// lib/libampcor/correlators.h): forward to the reference tree, found through -I <reference>/lib.
#include <libampcor/correlators.h>
