// Drop-in replacement for a MNMGDatalog driver's common/hash_table.cu:
// get_hash_table() is provided by libmnmgdl (include/mnmgdl_compat.h).
#include "mnmgdl_compat.h"
