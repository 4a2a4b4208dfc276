// Where the reference's sources include <ampcor/dom.h> (the installed name of
// lib/libampcor/dom.h): forward to the reference tree, found through -I <reference>/lib.
#include <libampcor/dom.h>
