/* ORACLE test infrastructure: the FreeSASA declarations the reference's swarm placement names
 * (used there only when the swarm count is 0).  Not called on the paths the harness drives;
 * anm_harness.cc defines them to abort the process. */
#pragma once
#include <stdio.h>
typedef struct freesasa_result { double total; } freesasa_result;
typedef struct freesasa_structure freesasa_structure;
typedef struct freesasa_node freesasa_node;
freesasa_structure* freesasa_structure_new(void);
freesasa_structure* freesasa_structure_from_pdb(FILE* pdb, const void* classifier, int options);
int freesasa_structure_n(const freesasa_structure* s);
freesasa_result* freesasa_calc_structure(const freesasa_structure* s, const void* parameters);
