/*
 * libdfb -- plain data types shared by the C ABI (dfb.h) and the device kernels:
 * error codes and the two sides of a Rys task.  Kept apart from the function
 * declarations so that the kernels do not depend on them.
 */
#ifndef DFB_TYPES_H
#define DFB_TYPES_H

#define DFB_OK 0
#define DFB_ERR_INVALID (-1)
#define DFB_ERR_CUDA (-2)
#define DFB_ERR_UNSUPPORTED (-3)
#define DFB_ERR_NOT_INITIALISED (-4)

/* AB side of a Rys task: AO shell pairs (A,B), or aux self-pairs (P, dummy). */
typedef struct {
    const int *shA, *shB;          /* per pair: shell indices in the AB basis (shB unused if b_dummy) */
    const int *pstart, *npair;     /* per pair: primitive-pair range in the tables below */
    const double *eta, *Px, *Py, *Pz, *cK;  /* per primitive pair */
    const double *ea, *eb;         /* per primitive pair: exponents of the A and B primitives */
    const double *cxyz;            /* AB basis shell centres (nshell, 3) */
    const int *aostart;            /* AB basis first function of each shell */
    const int *atom;               /* AB basis shell -> atom */
    int b_dummy;                   /* 1: B is the dummy s shell (metric) */
} dfb_pair_side_t;

/* C side of a Rys task: one aux shell (the dummy D is implicit). */
typedef struct {
    const double *cxyz;
    const int *pstart, *nprim;
    const double *pexp, *pcoef;
    const double *rexp;            /* 1 / pexp per primitive (the kernels' inner loops divide by nothing) */
    const int *aostart;
    const int *atom;
} dfb_aux_side_t;

#endif /* DFB_TYPES_H */
