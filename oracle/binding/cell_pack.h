/* cell_pack.c: the reference's cell block <-> the library's row layout. */
#ifndef CELL_PACK_H
#define CELL_PACK_H
struct Cell;
struct Sim;
int cell_pack_count(struct Sim *s);
void cell_pack(struct Cell ***c, struct Sim *s, double *prim, double *tiph, double *dphi);
void cell_unpack(struct Cell ***c, struct Sim *s, const double *prim, const double *cons, const double *tiph,
                 const double *dphi);
#endif
