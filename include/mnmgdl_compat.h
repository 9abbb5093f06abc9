/*
 * mnmgdl_compat.h -- the reference's operator signatures on top of libmnmgdl.
 *
 * C++ only. Include it where a MNMGDatalog driver includes
 * common/hash_table.cu and common/join.cu (after common/utils.cu has defined
 * `struct Entity {int key; int value;}`): the three functions below keep the
 * reference's names, argument meaning, ownership (results are cudaMalloc'd
 * buffers the caller cudaFree's) and error behaviour (print and exit(code) on
 * a failure, like checkCuda in common/error_handler.cu:1-7).
 *
 *   get_hash_table   common/hash_table.cu:24-55
 *   get_join         common/join.cu:51-87
 *   get_join_nl      common/join.cu:144-180
 *
 * The returned "hash table" is the library's index (a header, 16-byte slots
 * and the values of the key-sorted relation in one allocation); *hash_table_size
 * is its slot count. Work runs on the legacy default stream, as in the
 * reference; compute_time is host wall time like MPI_Wtime.
 */
#ifndef MNMGDL_COMPAT_H
#define MNMGDL_COMPAT_H

#include "mnmgdl.h"

extern "C" {
DL_API dl_entity *dl_compat_get_hash_table(int grid_size, int block_size, dl_entity *relation, int relation_size,
                                           int *hash_table_size, double *compute_time);
DL_API dl_entity *dl_compat_get_join(int grid_size, int block_size, dl_entity *hash_table, int hash_table_size,
                                     dl_entity *relation, int relation_size, int *join_result_size,
                                     double *compute_time);
DL_API dl_entity *dl_compat_get_join_nl(int grid_size, int block_size, dl_entity *sorted_relation,
                                        int sorted_relation_size, dl_entity *relation, int relation_size,
                                        int *join_result_size, double *compute_time);
}

inline Entity *get_hash_table(int grid_size, int block_size, Entity *edge, int edge_size, int *hash_table_size,
                              double *compute_time) {
    return reinterpret_cast<Entity *>(dl_compat_get_hash_table(grid_size, block_size,
                                                               reinterpret_cast<dl_entity *>(edge), edge_size,
                                                               hash_table_size, compute_time));
}

inline Entity *get_join(int grid_size, int block_size, Entity *hash_table, int hash_table_size, Entity *relation,
                        int relation_size, int *join_result_size, double *compute_time) {
    return reinterpret_cast<Entity *>(dl_compat_get_join(grid_size, block_size,
                                                         reinterpret_cast<dl_entity *>(hash_table), hash_table_size,
                                                         reinterpret_cast<dl_entity *>(relation), relation_size,
                                                         join_result_size, compute_time));
}

inline Entity *get_join_nl(int grid_size, int block_size, Entity *sorted_relation, int sorted_relation_size,
                           Entity *relation, int relation_size, int *join_result_size, double *compute_time) {
    return reinterpret_cast<Entity *>(dl_compat_get_join_nl(
        grid_size, block_size, reinterpret_cast<dl_entity *>(sorted_relation), sorted_relation_size,
        reinterpret_cast<dl_entity *>(relation), relation_size, join_result_size, compute_time));
}

#endif
