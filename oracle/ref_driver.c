/*
 * ref_driver.c -- TEST INFRASTRUCTURE, NOT PRODUCT CODE.
 *
 * Plain-C entry points over raw pointers that drive GPAW's own, unmodified
 * C kernels (c/bmgs/bmgs.c and c/bc.c, compiled from the reference tree by
 * oracle/Makefile into oracle/_ref/libgpawref.so).  The Python C-API layer
 * of the reference (c/operators.c, c/transformers.c) cannot be compiled for
 * Python 3, so its band loops are restated here without Python objects:
 *
 *   ref_fd_apply    <- Operator_apply + apply_worker   c/operators.c:316-405, 109-157
 *   ref_relax       <- Operator_relax                  c/operators.c:49-91
 *   ref_transform   <- Transformer_apply + transapply_worker
 *                                                      c/transformers.c:127-185, 54-123
 *
 * Bands are split over pthreads in contiguous chunks as in the GPAW_OMP
 * build of the reference (c/operators.c:116-124, c/transformers.c:67-75).
 * Phases are complex doubles laid out as phase_cd[3][2].
 */
#include <stdlib.h>
#include <string.h>
#include <pthread.h>
#include <complex.h>
#include "bc.h"

typedef struct {
  /* common */
  boundary_conditions* bc;
  int real;
  int nin;
  int nthds;
  int thread_id;
  const double* in;
  double* out;
  const double_complex* ph;
  /* operator */
  const bmgsstencil* stencil;
  /* transformer */
  int interpolate;
  int k;
  int (*skip)[2];
  int out_ng;
} ref_job;

static void band_range(const ref_job* j, int* b0, int* b1) {
  int per = j->nin / j->nthds, rem = j->nin % j->nthds;
  *b0 = j->thread_id * per + (j->thread_id < rem ? j->thread_id : rem);
  *b1 = *b0 + per + (j->thread_id < rem ? 1 : 0);
}

static void* fd_worker(void* arg) {
  ref_job* j = (ref_job*)arg;
  boundary_conditions* bc = j->bc;
  int ng = bc->ndouble * bc->size1[0] * bc->size1[1] * bc->size1[2];
  int ng2 = bc->ndouble * bc->size2[0] * bc->size2[1] * bc->size2[2];
  double* sendbuf = (double*)malloc(sizeof(double) * (bc->maxsend + 1));
  double* recvbuf = (double*)malloc(sizeof(double) * (bc->maxrecv + 1));
  double* buf = (double*)malloc(sizeof(double) * ng2);
  MPI_Request recvreq[2], sendreq[2];
  int b0, b1;
  band_range(j, &b0, &b1);
  for (int n = b0; n < b1; n++) {
    const double* in = j->in + (size_t)n * ng;
    double* out = j->out + (size_t)n * ng;
    for (int i = 0; i < 3; i++) {
      bc_unpack1(bc, in, buf, i, recvreq, sendreq, recvbuf, sendbuf,
                 j->ph ? j->ph + 2 * i : 0, j->thread_id, 1);
      bc_unpack2(bc, buf, i, recvreq, sendreq, recvbuf, 1);
    }
    if (j->real)
      bmgs_fd(j->stencil, buf, out);
    else
      bmgs_fdz(j->stencil, (const double_complex*)buf, (double_complex*)out);
  }
  free(buf); free(recvbuf); free(sendbuf);
  return NULL;
}

static void run_jobs(ref_job* proto, void* (*fn)(void*)) {
  int nthds = proto->nthds < 1 ? 1 : proto->nthds;
  if (nthds > proto->nin && proto->nin > 0) nthds = proto->nin;
  proto->nthds = nthds;
  ref_job* jobs = (ref_job*)malloc(sizeof(ref_job) * nthds);
  pthread_t* th = (pthread_t*)malloc(sizeof(pthread_t) * nthds);
  for (int t = 0; t < nthds; t++) { jobs[t] = *proto; jobs[t].thread_id = t; }
  for (int t = 1; t < nthds; t++) pthread_create(&th[t], NULL, fn, &jobs[t]);
  fn(&jobs[0]);
  for (int t = 1; t < nthds; t++) pthread_join(th[t], NULL);
  free(jobs); free(th);
}

/* coefs[P], flat offsets[P] on the padded grid, size[3], range (padding on
 * every face), neighbors[3][2] (0 = self/periodic, -1 = none). */
int ref_fd_apply(int P, const double* coefs, const long* offsets, const long size[3],
                 int range, const long neighbors[6], int real, int cfd, int nin,
                 const double* in, double* out, const double* phases, int nthreads) {
  bmgsstencil s = bmgs_stencil(P, coefs, offsets, range, size);
  const long padding[3][2] = {{range, range}, {range, range}, {range, range}};
  boundary_conditions* bc = bc_init(size, padding, padding,
                                    (const long (*)[2])neighbors, MPI_COMM_NULL, real, cfd);
  ref_job j;
  memset(&j, 0, sizeof(j));
  j.bc = bc; j.real = real; j.nin = nin; j.nthds = nthreads;
  j.in = in; j.out = out; j.stencil = &s;
  j.ph = real ? 0 : (const double_complex*)phases;
  if (nin > 0) run_jobs(&j, fd_worker);
  free(bc);
  bmgs_deletestencil(&s);
  return 0;
}

int ref_relax(int relax_method, int P, const double* coefs, const long* offsets,
              const long size[3], int range, const long neighbors[6], int cfd, double* fun,
              const double* src, int nrelax, double w) {
  bmgsstencil s = bmgs_stencil(P, coefs, offsets, range, size);
  const long padding[3][2] = {{range, range}, {range, range}, {range, range}};
  /* The operator's own boundary object: cfd = 0 for stencils with cross
     terms (gpaw/fd_operators.py:26-30), so corners are filled. */
  boundary_conditions* bc = bc_init(size, padding, padding,
                                    (const long (*)[2])neighbors, MPI_COMM_NULL, 1, cfd);
  const int* size2 = bc->size2;
  double* buf = (double*)malloc(sizeof(double) * size2[0] * size2[1] * size2[2]);
  double* sendbuf = (double*)malloc(sizeof(double) * (bc->maxsend + 1));
  double* recvbuf = (double*)malloc(sizeof(double) * (bc->maxrecv + 1));
  MPI_Request recvreq[2], sendreq[2];
  for (int n = 0; n < nrelax; n++) {
    for (int i = 0; i < 3; i++) {
      bc_unpack1(bc, fun, buf, i, recvreq, sendreq, recvbuf, sendbuf, 0, 0, 1);
      bc_unpack2(bc, buf, i, recvreq, sendreq, recvbuf, 1);
    }
    bmgs_relax(relax_method, &s, buf, fun, src, w);
  }
  free(recvbuf); free(sendbuf); free(buf); free(bc);
  bmgs_deletestencil(&s);
  return 0;
}

static void* tr_worker(void* arg) {
  ref_job* j = (ref_job*)arg;
  boundary_conditions* bc = j->bc;
  int ng = bc->ndouble * bc->size1[0] * bc->size1[1] * bc->size1[2];
  int ng2 = bc->ndouble * bc->size2[0] * bc->size2[1] * bc->size2[2];
  double* sendbuf = (double*)malloc(sizeof(double) * (bc->maxsend + 1));
  double* recvbuf = (double*)malloc(sizeof(double) * (bc->maxrecv + 1));
  double* buf = (double*)malloc(sizeof(double) * ng2);
  int buf2size = j->interpolate ? ng2 * 16 : ng2 / 2;
  double* buf2 = (double*)malloc(sizeof(double) * buf2size);
  MPI_Request recvreq[2], sendreq[2];
  int b0, b1;
  band_range(j, &b0, &b1);
  for (int n = b0; n < b1; n++) {
    const double* in = j->in + (size_t)n * ng;
    double* out = j->out + (size_t)n * j->out_ng;
    for (int i = 0; i < 3; i++) {
      bc_unpack1(bc, in, buf, i, recvreq, sendreq, recvbuf, sendbuf,
                 j->ph ? j->ph + 2 * i : 0, j->thread_id, 1);
      bc_unpack2(bc, buf, i, recvreq, sendreq, recvbuf, 1);
    }
    if (j->real) {
      if (j->interpolate)
        bmgs_interpolate(j->k, j->skip, buf, bc->size2, out, buf2);
      else
        bmgs_restrict(j->k, buf, bc->size2, out, buf2);
    } else {
      if (j->interpolate)
        bmgs_interpolatez(j->k, j->skip, (double_complex*)buf, bc->size2,
                          (double_complex*)out, (double_complex*)buf2);
      else
        bmgs_restrictz(j->k, (double_complex*)buf, bc->size2, (double_complex*)out,
                       (double_complex*)buf2);
    }
  }
  free(buf2); free(buf); free(recvbuf); free(sendbuf);
  return NULL;
}

/* Arguments as the reference Transformer constructor (c/transformers.c:222-265):
 * size_in[3], size_out[3], k, paddings[3][2], npaddings[3][2], skip[3][2],
 * neighbors[3][2], real, interpolate; then the apply arguments. */
int ref_transform(const long size_in[3], const long size_out[3], int k, const long pad[6],
                  const long npad[6], const long skip[6], const long neighbors[6], int real,
                  int interpolate, int nin, const double* in, double* out,
                  const double* phases, int nthreads) {
  boundary_conditions* bc = bc_init(size_in, (const long (*)[2])pad, (const long (*)[2])npad,
                                    (const long (*)[2])neighbors, MPI_COMM_NULL, real, 0);
  int sk[3][2];
  for (int c = 0; c < 3; c++)
    for (int d = 0; d < 2; d++) sk[c][d] = (int)skip[2 * c + d];
  ref_job j;
  memset(&j, 0, sizeof(j));
  j.bc = bc; j.real = real; j.nin = nin; j.nthds = nthreads;
  j.in = in; j.out = out; j.interpolate = interpolate; j.k = k; j.skip = sk;
  j.out_ng = bc->ndouble * (int)(size_out[0] * size_out[1] * size_out[2]);
  j.ph = real ? 0 : (const double_complex*)phases;
  if (nin > 0) run_jobs(&j, tr_worker);
  free(bc);
  return 0;
}
