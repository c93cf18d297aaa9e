/*
 * ORACLE - test infrastructure only.  A plain-C restatement of the reference's ERI algorithm
 * (McMurchie-Davidson / SHARK, src/lible/ints of MihkuU/Lible) used to check the CUDA engine.
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may load it.
 */
#ifndef ERI_PORT_H
#define ERI_PORT_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct port_mol port_mol;

/* Shells per atom in basis-file order; coordinates in bohr. */
port_mol *port_new(int n_atoms, const int *Z, const double *xyz_bohr, const int *shells_per_atom,
                   const int *shell_l, const int *shell_nprim, const double *exps, const double *coeffs);
void port_free(port_mol *m);
int port_nao(const port_mol *m);

/* Boys function F_0..F_n at x (src/lible/ints/boys_function.cpp:71-118). */
void port_boys(int n, double x, double *F);
/* Full (N^4) ERI tensor. */
void port_eri4(const port_mol *m, double *out);
/* Direct J/K over unique quartets with Schwarz threshold; every bra_stride-th bra pair.
 * Returns the number of quartets processed. */
long long port_jk(const port_mol *m, const double *D, double *J, double *K, double schwarz, int bra_stride);
/* Gradient of 1/2 Tr(DJ) - 1/4 Tr(DK), [n_atoms][3]. */
void port_jk_grad(const port_mol *m, const double *D, double *grad);

#ifdef __cplusplus
}
#endif
#endif
