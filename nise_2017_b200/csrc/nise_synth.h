/* Seeded synthetic NISE trajectories in the reference's binary layout (synth.c). */
#ifndef NISE_SYNTH_H
#define NISE_SYNTH_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

enum { NISE_SYNTH_CHAIN = 0, NISE_SYNTH_LATTICE = 1, NISE_SYNTH_CLUSTER = 2 };
enum { NISE_SYNTH_FULL = 0, NISE_SYNTH_COUPLING = 1 };

typedef struct {
    int n_sites;
    int frames;
    float dt_fs;
    int geometry;      /* NISE_SYNTH_CHAIN / _LATTICE / _CLUSTER */
    float spacing;     /* Angstrom: chain/lattice spacing; cluster mean spacing */
    float eps0;        /* mean site energy, cm^-1 */
    float sigma;       /* OU standard deviation, cm^-1 */
    float tau_fs;      /* OU correlation time, fs */
    float j_nn;        /* chain: mean nearest-neighbour coupling, cm^-1 */
    float j_sigma;     /* chain: per-frame Gaussian noise on j_nn, cm^-1 */
    float jcut;        /* point-dipole couplings below |jcut| are written as 0 */
    float mu_jitter;   /* per-frame Gaussian jitter per dipole component (Debye) */
    int ham_type;      /* NISE_SYNTH_FULL or NISE_SYNTH_COUPLING */
    int dipole_frames; /* dipole records to write (<=0: one per frame) */
    float anharm_mean, anharm_sigma; /* Anharmonicfile statistics, cm^-1 */
    uint64_t seed;
} nise_synth_spec;

/* Floats per energy record (without the int32 tag). */
long nise_synth_energy_record_floats(const nise_synth_spec *sp);
/* Fill caller buffers with record images; any buffer but energy may be NULL. */
int nise_synth_fill(const nise_synth_spec *sp, void *energy, void *dipole, void *coupling, void *anharm,
                    void *overtone);
/* Write the files; NULL paths are skipped (energy and dipole are required). */
int nise_synth_write(const nise_synth_spec *sp, const char *energy_path, const char *dipole_path,
                     const char *coupling_path, const char *anharm_path, const char *overtone_path);

#ifdef __cplusplus
}
#endif
#endif
