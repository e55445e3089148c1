/* remc_post.h - batched GPU post-processing of bound conformations and
 * trajectories (the reference's post processor, run over many frames at once).
 *
 * Both entry points take host buffers, run on the current CUDA device and
 * return REMC_OK (0) or a negative status; remc_last_error_string() (in
 * remc_b200.h) gives the message.
 *
 * Counterparts in the reference (iantunbridge/RemcDockingSimulator):
 *   remc_post_rebuild ... the pose reconstruction loop of pdbgen
 *                         (post processor/pdbgensrc/pdbgen.cpp:166-215):
 *                         Quaternion::normalize, Molecule::setRotation,
 *                         the image shift toward molecule 0,
 *                         Molecule::setPosition
 *   remc_post_drms ...... DRMS(Replica*, Replica*, bool)
 *                         (post processor/pdbgensrc/drms.cpp:7-57) and the
 *                         contact counts of DRMS(Replica*, Replica*)
 *                         (simulation engine/src/main.cpp:789-836)
 */
#ifndef REMC_POST_H
#define REMC_POST_H

#ifdef __cplusplus
extern "C" {
#endif

/* Rebuild bead coordinates from molecule poses.
 *   rel0[3 * n_beads]      bead positions relative to their molecule's centre
 *                          as loaded from the PDB files (Residue::relativePosition)
 *   mol_start[n_mol + 1]   first bead of every molecule
 *   shift[n_mol]           1: place the molecule's centre at the periodic image
 *                          nearest molecule 0's position (pdbgen does this for
 *                          non-crowders); 0: keep it
 *   centre0[3]             molecule 0's centre as loaded (its own image shift
 *                          is taken against this)
 *   box                    periodic box edge
 *   quat[n_frames][n_mol][4] rotation (w, x, y, z) of every molecule, as
 *                          written to _boundconformations
 *   centre[n_frames][n_mol][3] its centre
 *   pos[n_frames][n_beads][3] out: q.rotateVector(rel0) + centre', FP32
 *   centre_out[n_frames][n_mol][3] out (may be NULL): the shifted centres */
int remc_post_rebuild(const float* rel0, const int* mol_start, int n_mol, const int* shift,
                      const float* centre0, float box, const double* quat, const float* centre,
                      int n_frames, float* pos, float* centre_out);

/* Distance RMS of frames against a reference conformation: the mean over all
 * bead pairs (i, j) of different molecules I < J of
 * | |x_i - x_j| - |r_i - r_j| |, with FP32 distances and an FP64 sum.
 * reverse = 1 also evaluates the pairing with the reference's molecule order
 * swapped within each pair and keeps the smaller value (all molecules must
 * then have the same length). Contact counts per frame (any output may be
 * NULL): native = pairs with |r_i - r_j| < native_cut, recovered = native
 * pairs with |x_i - x_j| < recovered_cut, binding = pairs with
 * |x_i - x_j| < native_cut.
 *   frames[n_frames][n_beads][3], ref[n_beads][3], mol_start[n_mol + 1] */
int remc_post_drms(const float* frames, int n_frames, const float* ref, const int* mol_start,
                   int n_mol, int reverse, float native_cut, float recovered_cut, double* drms,
                   long long* native, long long* recovered, long long* binding);

#ifdef __cplusplus
}
#endif
#endif
