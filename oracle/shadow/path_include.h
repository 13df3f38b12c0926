/* Test infrastructure: the configure-time header of the reference's build (its CMake writes
 * source/dock/include/path_include.h from path_include.h.in), generated for the drop-in test so
 * that prepare_gso_tasks reads its DFIRE table from ./data/DCparams of the run directory. */
#pragma once
#define PROJECT_PATH "."
