/* Test-harness shim: the reference's src/graph.cpp includes <mpi.h> for its
 * multi-process path (graph.cpp:568-620), which the oracle never calls.  No
 * MPI is installed here, so this empty header lets that translation unit
 * compile.  Test infrastructure only; not part of the engine. */
#pragma once
