// Drop-in replacement for a MNMGDatalog driver's common/join.cu:
// get_join() and get_join_nl() are provided by libmnmgdl (include/mnmgdl_compat.h).
#include "mnmgdl_compat.h"
