/*
 * gviz_oracle.h -- CPU restatement of gviz's force-layout step (FP64).
 *
 * TEST INFRASTRUCTURE ONLY: the checker for libgvizcuda. Nothing in the
 * product (grapher_b200/, include/) includes or links this.
 * See gviz_oracle.c for the reference file:line each function follows.
 */
#ifndef GVIZ_ORACLE_H
#define GVIZ_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#define ORC_MODEL_FR 0
#define ORC_MODEL_LINLOG 1
#define ORC_DIR_TABLE 256

/* Same field meaning as gvizForceEmbedderState's configuration
 * (include/embedders/gvizForceEmbedder.h:52-125). */
typedef struct orcParams {
  int32_t model;
  int32_t barnesHutEnabled;
  int32_t preventOverlap;
  int32_t _pad;
  uint64_t nodesPerCell;
  double edgeLength;
  double theta;
  double gravityK;
  double radiusBase;
  double radiusPerDegree;
  double overlapConstant;
  double jitterTolerance;
} orcParams;

void orc_dir_table(double *out);
void orc_coincident_dir(uint64_t self, uint64_t other, double *ux, double *uy);

int orc_quadtree_leaves(const double *pts, const double *mass, size_t n,
                        size_t k, int32_t *leafDepth, uint64_t *pathHi,
                        uint64_t *pathLo, size_t *nodeCountOut);
size_t orc_quadtree_nodes(const double *pts, const double *mass, size_t n,
                          size_t k, size_t cap, int32_t *depth,
                          uint64_t *pathHi, uint64_t *pathLo, double *outMass,
                          double *comX, double *comY, int32_t *isLeaf,
                          uint64_t *count);

int orc_forces(size_t V, const uint64_t *rowOff, const uint32_t *cols,
               const double *mass, const uint64_t *degree, const orcParams *p,
               const double *pos, double *disp, double *structForce,
               double *attMag, double *repMag, uint64_t *interactions);

double orc_step(size_t V, const uint64_t *rowOff, const uint32_t *cols,
                const double *mass, const uint64_t *degree, const orcParams *p,
                double *pos, double *structForce, double *speedState,
                double *stats, double *dispOut, double *attMagOut,
                double *repMagOut, double *swingOut, double *tractionOut,
                double *appliedOut);

void orc_exact_repulsion(size_t V, const double *mass, const uint64_t *degree,
                         const orcParams *p, const double *pos,
                         const uint64_t *targets, size_t nTargets,
                         double *repOut);

void orc_pair_fr_att(const double *v, const double *u, double k, double *acc);
void orc_pair_fr_rep(const double *v, const double *u, double k,
                     double radiusSum, double overlapC, double *acc);
void orc_pair_linlog_att(const double *v, const double *u, double *acc);
void orc_pair_linlog_rep(const double *v, const double *u, double vm,
                         double om, double radiusSum, double overlapC,
                         double *acc);

#endif
