// iparts::integer_partitions (drop-in for the reference's
// modules/integer_partitions.h); implemented in liblemc.so.
#ifndef LAUGHLINEDGE_INTEGER_PARTITIONS_H
#define LAUGHLINEDGE_INTEGER_PARTITIONS_H
#include "lemc_api_core.h"
#endif
