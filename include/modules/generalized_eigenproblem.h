// ges::generalizedEigenproblem (drop-in for the reference's
// modules/generalized_eigenproblem.h); FP64, implemented in liblemc.so.
#ifndef LAUGHLINEDGE_GENERALIZED_EIGENPROBLEM_H
#define LAUGHLINEDGE_GENERALIZED_EIGENPROBLEM_H
#include "lemc_api_core.h"
#endif
