/*
 * kfun3d_b200: the GEOMETRY record the reference's kernels take.
 *
 * The drop-in entry points in kfun3d_b200.h keep the reference's signatures
 * (inc/core_kernel.h:6-22), so this record must have exactly the layout of the
 * reference's inc/geometry.h:1-107: same members, same order, same types
 * (unsigned long int is 64-bit on LP64).  A GEOMETRY built by the reference's
 * Setup (src/mesh.c:22-154) and one built by kfun3d_setup_load() are
 * interchangeable.  When both headers are in one translation unit, include only
 * one of them; the guard below is the reference's own so that works.
 */
#ifndef __FUN3D_INC_GEOMETRY_H
#define __FUN3D_INC_GEOMETRY_H

struct xyzn {          /* per edge: unit normal (x0,x1,x2) n0->n1 and dual-face area x3 */
  double *x0;
  double *x1;
  double *x2;
  double *x3;
};

struct xyz {           /* three coordinate arrays; also the gradient (GRADIENT) */
  double *x0;
  double *x1;
  double *x2;
};

typedef struct xyz GRADIENT;

struct edge {          /* 0-based end points, edges sorted by n0 */
  unsigned int *n0;
  unsigned int *n1;
};

struct face {          /* wall triangles, global node ids */
  unsigned int *n0;
  unsigned int *n1;
  unsigned int *n2;
};

struct weights {       /* least-squares terms: w0 used at n0, w1 at n1 */
  struct xyz *w0;
  struct xyz *w1;
};

struct etbl {
  unsigned long int sz;
  struct edge *eptr;
  struct xyzn *xyzn;
  struct weights *w;
};

struct ntbl {
  unsigned long int sz;
  struct xyz *xyz;
  unsigned int *part;  /* owning OpenMP thread of each node */
  double *cdt;         /* local pseudo-time diagonal */
};

struct stbl {
  unsigned long int sz;
  unsigned int *i;     /* sz+1 offsets */
};

struct bntbl {         /* boundary nodes: global id and node normal (magnitude = area) */
  unsigned long int sz;
  unsigned int *nptr;
  struct xyz *xyz;
};

struct bftbl {
  unsigned long int sz;
  struct face *fptr;
};

struct btbl {
  struct bntbl *s;     /* slip-wall nodes */
  struct bntbl *f;     /* far-field nodes */
  struct bftbl *fc;    /* wall faces, grouped by colour */
};

struct ctbl {
  unsigned int b;      /* block size, 4 */
  unsigned int b2;
  unsigned long int sz;/* 4 * nodes */
};

struct qtbl {
  double *q;           /* state, q[4*node + var], var = p,u,v,w */
};

typedef struct geometry {
  struct etbl *e;      /* edges */
  struct ntbl *n;      /* nodes */
  struct btbl *b;      /* boundaries */
  struct ctbl *c;      /* block sizes */
  struct stbl *s;      /* per-thread edge ranges (s->sz threads) */
  struct stbl *t;      /* wall-face colour offsets (t->sz colours) */
  struct qtbl *q;      /* state */
  void *matrix;        /* opaque matrix handle (CXX_Matrix_Init) */
} GEOMETRY;

#endif /* __FUN3D_INC_GEOMETRY_H */
