/* gazpart_files.h -- the reference's particle files, read and written natively.
 *
 * The reference writes its particle restart and snapshot files with Fortran
 * sequential unformatted I/O (gfortran, native little-endian, 4-byte record markers).
 * A logical record of L bytes is stored as one or more subrecords
 *     [int32 head][data][int32 tail]
 * of at most 2147483639 data bytes each (gfortran's default maximum subrecord
 * length).  head = tail = the subrecord's data length, except that the head is
 * negated when more subrecords of the same record follow and the tail is negated
 * when subrecords of the same record precede it.  A record of L <= 2147483639 bytes
 * is therefore the plain [L][data][L].
 *
 * Files (column order x y z u v w qa qb qc qd ox oy oz, as GP_NSTATE, then IDP):
 *  - class restart, SAVE_PARTICLE with ISAVEPART = 2 (save_particle.f90:116-180) and
 *    its reader INITIATION_PARTICLE_POSITION (initiation_particle_position.f90:430-532):
 *      NPART_FULL (int32) | NPCLASS(J,:) (int32[pd]) | RHOP(J,:) (f64[pd])
 *      | EMAJ_PART(J,:) (f64[pd]) | APR_PART(J) (f64) | 14 records of NPART_FULL f64
 *    with the 14th column real(IDP).  Named part_pJJ_tNNNNNNNN.bin, part_pJJ.end, and
 *    read back as part_pJJ.ini.
 *  - snapshot, PRINT_PARTICLE (print_particle.f90:145-170): the same 14 records
 *    without the header.
 *
 * All functions return a GP_* status (gazpart_gpu.h). */
#ifndef GAZPART_FILES_H
#define GAZPART_FILES_H

#include <stdint.h>

#include "gazpart_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

#define GP_NPARTCOL 14              /* columns of the class restart and snapshot files */
#define GP_FUNF_MAX_SUBRECORD 2147483639LL

/* Generic sequential unformatted file.  writing = 0 opens an existing file for
 * reading, 1 creates or replaces one (Fortran status='replace'). */
typedef struct gp_funf gp_funf;
int gp_funf_open(const char *path, int32_t writing, gp_funf **f);
int gp_funf_close(gp_funf *f);
/* Largest subrecord written from now on (gfortran's -fmax-subrecord-length); between
 * 1 and GP_FUNF_MAX_SUBRECORD.  Readers accept any split. */
int gp_funf_set_max_subrecord(gp_funf *f, int64_t nbytes);
/* One Fortran WRITE statement of nbytes bytes: one logical record. */
int gp_funf_write(gp_funf *f, const void *data, int64_t nbytes);
/* Size of the next logical record without consuming it; GP_EEOF at the end. */
int gp_funf_record_size(gp_funf *f, int64_t *nbytes);
/* One Fortran READ statement: the first nbytes of the next record go to dst (NULL
 * with nbytes = 0 skips the record, as an empty READ does) and the rest of the record
 * is passed over.  A record shorter than nbytes gives GP_ERECORD and is consumed. */
int gp_funf_read(gp_funf *f, void *dst, int64_t nbytes);

/* Class restart file (ISAVEPART = 2).  cols: GP_NPARTCOL host columns of n doubles,
 * the last one real(IDP).  n must fit the reference's int32 NPART_FULL. */
int gp_write_part_class(const char *path, int64_t n, int32_t polydisp, const int32_t *npclass,
                        const double *rhop, const double *emaj, double apr, const double *const *cols);
/* The file's NPART_FULL and the length of its NPCLASS record in entries (POLYDISPMAX
 * of the run that wrote it). */
int gp_read_part_class_header(const char *path, int64_t *n, int32_t *polydisp);
/* Reads what INITIATION_PARTICLE_POSITION reads: polydisp table entries (at most the
 * file's) and n values of each column (n must equal the file's NPART_FULL). */
int gp_read_part_class(const char *path, int64_t n, int32_t polydisp, int32_t *npclass, double *rhop,
                       double *emaj, double *apr, double *const *cols);

/* Snapshot file (PRINT_PARTICLE): GP_NPARTCOL records of n doubles. */
int gp_write_part_snapshot(const char *path, int64_t n, const double *const *cols);
int gp_read_part_snapshot(const char *path, int64_t n, double *const *cols);

/* Class ig of a context straight to a class restart file: its state is downloaded in
 * the class's own particle order and written with the given tables.  idp: the
 * polydisperse index of each particle (host, n entries) or NULL for all 1. */
int gp_save_part_class(gp_ctx *ctx, int32_t ig, const char *path, int32_t polydisp, const int32_t *npclass,
                       const double *rhop, const double *emaj, double apr, const int32_t *idp);
/* A class restart file into a context as a new class on field slot `field`
 * (gp_add_class).  Each particle's constants follow from its IDP = int(column 14):
 * EMAJ = EMAJ_PART(J,IDP), APR = APR_PART(J), RHOP = RHOP(J,IDP) and the inertia
 * (b^2+c^2)/5, (a^2+c^2)/5, (a^2+b^2)/5 with b = c = a/APR
 * (initiation_particle_position.f90:609-624).  An IDP outside 1..polydisp gives
 * GP_EBADARG.  *n receives the particle count when n is not NULL. */
int gp_load_part_class(gp_ctx *ctx, const char *path, int32_t field, int32_t *ig, int64_t *n);

#ifdef __cplusplus
}
#endif
#endif /* GAZPART_FILES_H */
