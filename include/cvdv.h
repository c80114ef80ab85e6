/*
 * libcvdv (B200 build) -- C ABI of the dense CV-DV state-vector path.
 *
 * Drop-in for the reference CUDA-CVDV library: every function of the
 * reference's src/cuda/api.h:14-61 is exported here with the same name,
 * signature and argument meaning, so the reference's Python wrapper
 * (src/cudaCvdv.py:29-74, which binds them with ctypes) loads this library
 * unchanged.  Each declaration cites the reference entry point it replaces.
 *
 * Differences in error behaviour (the reference prints to stderr and returns,
 * or throws a C++ exception through the C ABI on CUDA failures):
 *   - no function here throws, traps or exits;
 *   - invalid arguments leave the state untouched and record an error that
 *     cvdvGetLastError() returns (the output buffers are not written, except
 *     where the reference writes 0: cvdvGetFidelity / cvdvFidelityStatevectors);
 *   - gates called before the state is initialised record an error instead of
 *     running on an empty buffer.
 *
 * Execution: gates are queued on the context and run, fused, at the next
 * readout (m / getState / Wigner / Husimi / fidelity / photon number / norm),
 * at cvdvSetStateFromDevicePtr, or at cvdvSynchronize.  All device work of a
 * context runs on one CUDA stream owned by the context; that stream is a
 * blocking stream, so it is ordered with work on the legacy default stream.
 * Readouts return after their results are on the host.  A context is not
 * thread-safe (as in the reference).
 */
#ifndef CVDV_B200_H
#define CVDV_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct CVDVContext CVDVContext;

/* ---------------------------------------------------------------- lifecycle */

/* src/cuda/context.cu:7-67 (api.h:14).  Registers: numQubits[r] >= 1 each,
 * sum <= 34.  complex128 state.  Returns NULL only if the host allocation
 * fails; a context created with bad sizes has no registers and records an
 * error. */
CVDVContext* cvdvCreate(int numReg, int* numQubits);
/* src/cuda/context.cu:70-72 (api.h:15). */
void cvdvDestroy(CVDVContext* ctx);
/* src/cuda/context.cu:117-129 (api.h:16): release device memory, keep the handle. */
void cvdvFree(CVDVContext* ctx);
/* src/cuda/context.cu:75-115 (api.h:17).  devicePtrs[r] points to N_r
 * complex128 values (device or host memory); psi = tensor product, last
 * register fastest, not normalised.  Built on the device, at the next flush
 * (cvdvSetFusion bit 4).  The arrays are copied on the context's stream, so the
 * caller's buffers must stay valid until that stream has run (cvdvSynchronize). */
void cvdvInitFromSeparable(CVDVContext* ctx, void** devicePtrs, int numReg);
/* src/cuda/context.cu:131-137 (api.h:18).  d_src: 2^n complex128 values
 * (device or host memory). */
void cvdvSetStateFromDevicePtr(CVDVContext* ctx, void* d_src);
/* src/cuda/context.cu:139-163 (api.h:19-23). */
int cvdvGetNumRegisters(CVDVContext* ctx);
size_t cvdvGetTotalSize(CVDVContext* ctx);
void cvdvGetRegisterInfo(CVDVContext* ctx, int* qubitCountsOut, double* gridStepsOut);
int cvdvGetRegisterDim(CVDVContext* ctx, int regIdx);
double cvdvGetRegisterDx(CVDVContext* ctx, int regIdx);

/* ---------------------------------------------------------------- gates */

/* src/cuda/gates.cu:19-67 (api.h:25): centred DFT q -> p. */
void cvdvFtQ2P(CVDVContext* ctx, int regIdx);
/* src/cuda/gates.cu:69-122 (api.h:26): centred inverse DFT p -> q. */
void cvdvFtP2Q(CVDVContext* ctx, int regIdx);
/* src/cuda/gates.cu:124-161 (api.h:27). */
void cvdvDisplacement(CVDVContext* ctx, int regIdx, double betaRe, double betaIm);
/* src/cuda/gates.cu:163-204 (api.h:28-29). */
void cvdvConditionalDisplacement(CVDVContext* ctx, int targetReg, int ctrlReg, int ctrlQubit,
                                 double betaRe, double betaIm);
/* src/cuda/gates.cu:206-219 (api.h:30); axis 0/1/2 = X/Y/Z. */
void cvdvPauliRotation(CVDVContext* ctx, int regIdx, int qubitIdx, int axis, double theta);
/* src/cuda/gates.cu:221-233 (api.h:31). */
void cvdvHadamard(CVDVContext* ctx, int regIdx, int qubitIdx);
/* src/cuda/gates.cu:235-246 (api.h:32). */
void cvdvParity(CVDVContext* ctx, int regIdx);
/* src/cuda/gates.cu:248-268 (api.h:33). */
void cvdvConditionalParity(CVDVContext* ctx, int targetReg, int ctrlReg, int ctrlQubit);
/* src/cuda/gates.cu:270-286 (api.h:34). */
void cvdvSwapRegisters(CVDVContext* ctx, int reg1, int reg2);
/* src/cuda/gates.cu:288-300 (api.h:35): exp(i t q^2). */
void cvdvPhaseSquare(CVDVContext* ctx, int regIdx, double t);
/* src/cuda/gates.cu:302-314 (api.h:36): exp(i t q^3). */
void cvdvPhaseCubic(CVDVContext* ctx, int regIdx, double t);
/* src/cuda/gates.cu:316-348 (api.h:37). */
void cvdvRotation(CVDVContext* ctx, int regIdx, double theta);
/* src/cuda/gates.cu:350-392 (api.h:38-39). */
void cvdvConditionalRotation(CVDVContext* ctx, int targetReg, int ctrlReg, int ctrlQubit,
                             double theta);
/* src/cuda/gates.cu:394-421 (api.h:40). */
void cvdvSqueeze(CVDVContext* ctx, int regIdx, double r);
/* src/cuda/gates.cu:423-459 (api.h:41-42). */
void cvdvConditionalSqueeze(CVDVContext* ctx, int targetReg, int ctrlReg, int ctrlQubit,
                            double r);
/* src/cuda/gates.cu:461-502 (api.h:43). */
void cvdvBeamSplitter(CVDVContext* ctx, int reg1, int reg2, double theta);
/* src/cuda/gates.cu:504-547 (api.h:44-45). */
void cvdvConditionalBeamSplitter(CVDVContext* ctx, int reg1, int reg2, int ctrlReg, int ctrlQubit,
                                 double theta);
/* src/cuda/gates.cu:549-565 (api.h:46): exp(i coeff q1 q2). */
void cvdvQ1Q2Gate(CVDVContext* ctx, int reg1, int reg2, double coeff);

/* ---------------------------------------------------------------- readouts */

/* src/cuda/bosonic.cu:103-132 (api.h:48): native N x N Wigner, row = p. */
void cvdvGetWigner(CVDVContext* ctx, int regIdx, double* wignerOut);
/* src/cuda/bosonic.cu:134-138 (api.h:49): Husimi Q (overlap route, falling
 * back to the Wigner route under the same memory rule as the reference). */
void cvdvGetHusimiQ(CVDVContext* ctx, int regIdx, double* husimiOut);
/* src/cuda/bosonic.cu:140-144 (api.h:50). */
void cvdvGetHusimiQOverlap(CVDVContext* ctx, int regIdx, double* husimiOut);
/* src/cuda/bosonic.cu:146-150 (api.h:51). */
void cvdvGetHusimiQWigner(CVDVContext* ctx, int regIdx, double* husimiOut);
/* src/cuda/measure.cu:65-123 (api.h:53-54): joint marginal, first selected
 * register fastest. */
void cvdvMeasureMultiple(CVDVContext* ctx, const int* regIdxs, int numRegs, double* probsOut);
/* src/cuda/measure.cu:125-256 (api.h:55-56): same result as
 * cvdvMeasureMultiple (the reference computes it with cuTENSOR). */
void cvdvMeasureMultipleCT(CVDVContext* ctx, const int* regIdxs, int numRegs, double* probsOut);
/* src/cuda/measure.cu:258-274 (api.h:57). */
void cvdvGetState(CVDVContext* ctx, double* realOut, double* imagOut);
/* src/cuda/measure.cu:276-300 (api.h:58): sum |psi|^2 (not its square root). */
double cvdvGetNorm(CVDVContext* ctx);
/* src/cuda/measure.cu:302-318 (api.h:59): |<psi|prod_r phi_r>|^2. */
void cvdvGetFidelity(CVDVContext* ctx, void** devicePtrs, int numReg, double* fidOut);
/* src/cuda/measure.cu:320-331 (api.h:60): (<q^2> + <p^2> - 1) / 2.  The state
 * is not modified (the reference transforms it to p and back). */
double cvdvGetPhotonNumber(CVDVContext* ctx, int regIdx);
/* src/cuda/measure.cu:333-366 (api.h:61): |<psi1|psi2>|^2. */
void cvdvFidelityStatevectors(CVDVContext* ctx1, CVDVContext* ctx2, double* fidOut);

/* ---------------------------------------------------------------- extensions
 * No reference counterpart. */

/* Precision of the state: 0 = complex128 (plain, the default of cvdvCreate),
 * 1 = complex64 state with FP64 phase generation and FP64 reductions. */
CVDVContext* cvdvCreateEx(int numReg, int* numQubits, int precision);
int cvdvGetPrecision(CVDVContext* ctx);
/* Last error of ctx (or of the process when ctx is NULL): returns the code
 * (0 = none) and copies the message into msg[0..len). */
int cvdvGetLastError(CVDVContext* ctx, char* msg, int len);
void cvdvClearError(CVDVContext* ctx);
/* Run every queued gate and wait for the context's stream. */
void cvdvSynchronize(CVDVContext* ctx);
/* Run every queued gate without waiting (enqueue only). */
void cvdvFlush(CVDVContext* ctx);
/* Number of gate stages currently queued. */
int cvdvPendingStages(CVDVContext* ctx);
/* Device pointer to the live state (complex128 or complex64 per precision),
 * valid until the next gate flush; flushes first. */
void* cvdvGetStateDevicePtr(CVDVContext* ctx);
/* The context's CUDA stream (cudaStream_t). */
void* cvdvGetStream(CVDVContext* ctx);
/* Queue optimisations.  flags bit 0 (default on): an FtP2Q(r) followed by an
 * FtQ2P(r) (or the reverse) with only stages that leave register r untouched in
 * between is removed from the queue -- the pair is the identity, so the result
 * is unchanged up to rounding.  flags bit 1 (default on): consecutive 2x2 qubit
 * gates on up to five distinct qubits, with the diagonal runs between them, run
 * as one pass over the state instead of one pass per gate.  flags bit 2 (default
 * on): transforms of a register that is not the last one run as register-resident
 * column DFTs (one pass up to 2^8 points, two passes up to 2^16) instead of the
 * shared-memory tile passes.  flags bit 3 (default on): a run of transforms and
 * diagonal gates on such a register (2^8 .. 2^13 points, 2^14 in complex64) runs
 * as one pass with each column held on chip.  flags bit 4 (default on): after
 * cvdvInitFromSeparable on two or more registers, the queued stages that act on
 * one register of 2^8 .. 2^14 points alone, ahead of every stage that couples it
 * to another register, run on that register's array before the product is formed
 * (at the next flush).  flags bit 5 (default off): in complex64 contexts, the
 * transforms of a register that is not the last one, of 2^12 .. 2^14 points with
 * at least 32 amplitudes below it, run their two-pass (chained) column passes as
 * DFT-matrix products on the tensor cores (split-BF16 three-term products, FP32
 * accumulation, about 3e-6 relative error per 128-point DFT) instead of bit 3's
 * one-pass programs.  cvdvCancelledTransforms counts the transforms removed so
 * far. */
void cvdvSetFusion(CVDVContext* ctx, int flags);
long long cvdvCancelledTransforms(CVDVContext* ctx);
/* Number of kernels this library has launched in the process so far. */
unsigned long long cvdvLaunchCount(void);
/* Per-launch timing: when on, every kernel launch of ctx is bracketed by a CUDA
 * event pair.  cvdvGetKernelStats waits for the stream, returns the number of
 * kernel kinds, fills total milliseconds and launch counts per kind
 * (0 FFT pass, 1 qubit pair, 2 diagonal run, 3 permutation, 4 factor table,
 * 5 initialiser, 6 reduction, 7 phase space, 8 qubit-gate sequence, 9 column
 * transform pass) and resets
 * them. */
void cvdvSetTiming(CVDVContext* ctx, int on);
int cvdvGetKernelStats(CVDVContext* ctx, double* msOut, long long* countOut, int n);
/* Marginals of several single registers in one pass over the state:
 * probsOut receives, for each k, dims[regIdxs[k]] values back to back. */
void cvdvMeasureEach(CVDVContext* ctx, const int* regIdxs, int numRegs, double* probsOut);
/* ---------------------------------------------------------------- batched
 * variational circuits (no reference counterpart; the reference's TorchCvdv is
 * not differentiable in its gate parameters).  A batch is one caller-owned
 * device array of `batch` states of n qubits each (complex128 or complex64 per
 * precision, instance b at offset b 2^n), laid out [qubit registers..., mode]
 * with the mode the last register.  Each instance has its own parameter per
 * gate (device arrays of `batch` doubles).  Every call only enqueues work on
 * `stream` and returns 0 or an error code (message via cvdvGetLastError(NULL)).
 *
 * Rx(sign * thetas[b]) on flat bit `bit` of every instance. */
int cvdvBatchRx(void* states, int precision, int batch, int n, int bit, const double* thetas, double sign,
                void* stream);
/* cd(sign * betas[b]) with a real displacement (src/cuda/gates.cu:163-204) on a
 * mode of modeQubits (8..12) bits, controlled by flat bit ctrlBit. */
int cvdvBatchCondDisp(void* states, int precision, int batch, int n, int modeQubits, int ctrlBit,
                      const double* betas, double sign, void* stream);
/* Adjoint steps.  With psi the state after the gate and lam the back-propagated
 * target, write g_b = <lam_b| G |psi_b> (complex, gOut[2b], gOut[2b+1], device)
 * for the gate's generator G (Rx(theta) = exp(-i theta X/2): G = -X/2; cd(beta)
 * = exp(i beta G)) and apply the inverse gate to both arrays. */
int cvdvBatchRxAdjoint(void* psi, void* lam, int precision, int batch, int n, int bit, const double* thetas,
                       double* gOut, void* stream);
int cvdvBatchCondDispAdjoint(void* psi, void* lam, int precision, int batch, int n, int modeQubits,
                             int ctrlBit, const double* betas, double* gOut, void* stream);
/* A layer Rx(thetas[b]) on flat bit `bit` followed by cd(betas[b]) controlled by
 * the same bit, on a mode of modeQubits (9..12) bits, as one pass (a cluster of
 * two CTAs per pair of rows that differ in the bit).  Equal to cvdvBatchRx then
 * cvdvBatchCondDisp with sign +1. */
int cvdvBatchRxCondDisp(void* states, int precision, int batch, int n, int modeQubits, int bit,
                        const double* thetas, const double* betas, void* stream);
/* Adjoint of that layer: cvdvBatchCondDispAdjoint then cvdvBatchRxAdjoint in one
 * pass, writing g for the cd to gCd and for the Rx to gRx (as gOut above). */
int cvdvBatchRxCondDispAdjoint(void* psi, void* lam, int precision, int batch, int n, int modeQubits, int bit,
                               const double* thetas, const double* betas, double* gRx, double* gCd,
                               void* stream);
/* out[2b], out[2b+1] = <target| states_b> (target shared by every instance, or
 * one per instance when targetPerInstance != 0). */
int cvdvBatchOverlap(const void* states, const void* target, int precision, int batch, int n,
                     int targetPerInstance, double* out, void* stream);

/* ---------------------------------------------------------------- batched
 * independent circuits (no reference counterpart).  Many instances, each with
 * its own layout [1-qubit registers..., mode of 2^8..2^14 points] and its own
 * gate list, advance one gate per stage; one persistent launch runs every
 * instance's gate of a stage.  The host compiles each instance's gate into
 * tasks: a row program (the mode's transforms and diagonal phases, row by
 * row) or a qubit pair gate.  Diagonal phases are evaluated in-kernel:
 *   factor(j) = scale exp(i [tw theta_j + g0 + Z h0 + (a1 + Z b1) x + (a2 + Z b2) x^2 + a3 x^3])
 * with x = (j - (N-1)/2) dx, theta_j the transform twiddle pi (N-1)(2j-N+1)/(2N),
 * and Z = -1 when flat bit ctrlBit of the row is set (+1 otherwise or if -1). */
typedef struct {
  double a1, b1, a2, b2, a3, g0, h0, scale;
  int tw;
  int ctrlBit;
} CvdvBatchPhase;

typedef struct {
  int nOps;
  int op[15]; /* 0 next diagonal phase, 1 forward DFT, 2 inverse DFT (unnormalised), 3 parity */
  CvdvBatchPhase phase[8];
} CvdvBatchProgram;

typedef struct {
  long long stateOffset; /* first amplitude of the instance in the batch array */
  int kind;              /* 0 row program, 1 2x2 gate on a qubit bit */
  int n;                 /* qubits of the instance */
  int logRow;            /* qubits of its mode (row length) */
  int first;             /* first row (row program) or first pair (gate) */
  int count;             /* rows or pairs */
  int bit;               /* gate: flat bit */
  int program;           /* row program: index into the program table */
  int logE;              /* row program: log2 amplitudes per thread (3, 4 or 5: radix-8,
                            16 or 32 stages, 512 * 2^logE / 2^logRow rows per CTA);
                            0 = 5 for complex64 rows of 2^13 and more points, else 4 */
  double m[8];           /* gate: 2x2 matrix row-major, (re, im) pairs */
} CvdvBatchTask;

/* sizes[0..2] = sizeof(CvdvBatchPhase), sizeof(CvdvBatchProgram), sizeof(CvdvBatchTask) */
void cvdvBatchStructSizes(int* sizes);
/* Run one stage: tasks[0..nTasks) (device) over the batch array `states`
 * (complex128 or complex64), row programs from `programs` (device), on
 * gridCtas persistent CTAs of 512 threads; enqueue only. */
int cvdvBatchRunStage(void* states, int precision, const CvdvBatchTask* tasks, int nTasks,
                      const CvdvBatchProgram* programs, int gridCtas, void* stream);

/* Device-side separable register arrays (the input of cvdvInitFromSeparable), the
 * generators of src/cvdv.cu:187-295 and the setters of src/separable.py:44-132:
 * writes 2^numQubits complex128 values to the device array `out` on `stream`
 * (NULL = default stream), enqueue only.  kind / params:
 *   0 basis state {j0}; 1 uniform {}; 2 coherent {Re a, Im a};
 *   3 Fock {n}; 4 Fock superposition {Re c0, Im c0, Re c1, Im c1, ...};
 *   5 normalised sum of coherent states {Re a, Im a, Re c, Im c, ...};
 *   6 squeezed coherent D(a) S(r)|0> {r, Re a, Im a} (no reference setter).
 * At most 256 parameters.  Returns 0 or an error code (cvdvGetLastError(NULL, ..)). */
int cvdvSeparableFill(void* out, int numQubits, int kind, const double* params, int nParams, void* stream);

/* No counterpart in the reference.  The joint marginal of cvdvMeasureMultiple
 * for callers that cannot let the library allocate device memory (their device
 * memory belongs to another allocator, is fixed at start-up, or must not see
 * the device-wide synchronisation of cudaMalloc/cudaFree).  The caller passes
 * its own state (device memory of the current device, layout numQubits[0..numReg),
 * precision 0 = complex128 / 1 = complex64), its own device output probsOut of
 * prod 2^numQubits[regIdxs[k]] doubles, and a cudaStream_t (NULL = default
 * stream); the call only enqueues work and returns 0 or an error code (message
 * via cvdvGetLastError(NULL, ...)).  Partial histograms live in a fixed
 * 4.625 MiB device array that every GPU loading the library holds until exit,
 * so marginals are limited to 4096 outcomes (12 qubits); larger ones are
 * rejected.  The array and the two kernels live in the library's device code,
 * which CUDA loads on a device when it is first used (lazy module loading, the
 * default since CUDA 12.2); that load takes device memory (the array plus the
 * kernels' code).  cvdvCreate / cvdvCreateEx do it for their device, so after
 * any context was made on a device the first call allocates nothing.  In a
 * process that made none, the first call on a device does that set-up (load,
 * address lookup): make it before the caller's allocator takes the remaining
 * memory and before any stream capture.  All calls share the array: calls
 * that overlap on the GPU race. */
int cvdvMeasureMultipleNoAlloc(const void* state, int precision, const int* numQubits, int numReg,
                               const int* regIdxs, int numRegs, double* probsOut, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* CVDV_B200_H */
