/*
 * beagle_b200.h -- C ABI of the B200 (sm_100a) resource for BEAGLE's
 * phylogenetic-likelihood hot path.
 *
 * Every entry point is the beagle.h call of the same name with the prefix
 * "beagle" replaced by "beagleB200": same arguments, same meaning, same
 * return codes (0 = success, negative = BeagleB200ReturnCodes).  The comment
 * on each declaration cites the beagle.h declaration (libhmsbeagle/beagle.h,
 * beagle-lib 4.0.1) that it replaces.  Only plain C types cross this boundary:
 * host pointers owned by the caller and valid for the duration of the call.
 *
 * Flag bits, operation layouts and return codes have the numeric values of
 * beagle.h, so a beagle.h client passes its own values unchanged.
 *
 * The library runs on one CUDA device per instance (resourceList[0] picks the
 * device ordinal; default 0; entry k of beagleB200GetResourceList is device
 * k).  It has no CPU fallback: on a device other than sm_100,
 * beagleB200CreateInstance returns BEAGLE_B200_ERROR_NO_RESOURCE.
 */
#ifndef BEAGLE_B200_H
#define BEAGLE_B200_H

#ifdef __cplusplus
extern "C" {
#endif

/* Return codes: values of BeagleReturnCodes (beagle.h:110-122). */
enum BeagleB200ReturnCodes {
    BEAGLE_B200_SUCCESS = 0,
    BEAGLE_B200_ERROR_GENERAL = -1,
    BEAGLE_B200_ERROR_OUT_OF_MEMORY = -2,
    BEAGLE_B200_ERROR_UNIDENTIFIED_EXCEPTION = -3,
    BEAGLE_B200_ERROR_UNINITIALIZED_INSTANCE = -4,
    BEAGLE_B200_ERROR_OUT_OF_RANGE = -5,
    BEAGLE_B200_ERROR_NO_RESOURCE = -6,
    BEAGLE_B200_ERROR_NO_IMPLEMENTATION = -7,
    BEAGLE_B200_ERROR_FLOATING_POINT = -8
};

/* Capability flags: bit values of BeagleFlags (beagle.h:132-177). */
#define BEAGLE_B200_FLAG_PRECISION_SINGLE        (1L << 0)
#define BEAGLE_B200_FLAG_PRECISION_DOUBLE        (1L << 1)
#define BEAGLE_B200_FLAG_COMPUTATION_SYNCH       (1L << 2)
#define BEAGLE_B200_FLAG_COMPUTATION_ASYNCH      (1L << 3)
#define BEAGLE_B200_FLAG_EIGEN_REAL              (1L << 4)
#define BEAGLE_B200_FLAG_EIGEN_COMPLEX           (1L << 5)
#define BEAGLE_B200_FLAG_SCALING_MANUAL          (1L << 6)
#define BEAGLE_B200_FLAG_SCALING_AUTO            (1L << 7)
#define BEAGLE_B200_FLAG_SCALING_ALWAYS          (1L << 8)
#define BEAGLE_B200_FLAG_SCALERS_RAW             (1L << 9)
#define BEAGLE_B200_FLAG_SCALERS_LOG             (1L << 10)
#define BEAGLE_B200_FLAG_VECTOR_NONE             (1L << 12)
#define BEAGLE_B200_FLAG_THREADING_NONE          (1L << 14)
#define BEAGLE_B200_FLAG_PROCESSOR_GPU           (1L << 16)
#define BEAGLE_B200_FLAG_INVEVEC_STANDARD        (1L << 20)
#define BEAGLE_B200_FLAG_INVEVEC_TRANSPOSED      (1L << 21)
#define BEAGLE_B200_FLAG_FRAMEWORK_CUDA          (1L << 22)
#define BEAGLE_B200_FLAG_SCALING_DYNAMIC         (1L << 25)
#define BEAGLE_B200_FLAG_PARALLELOPS_STREAMS     (1L << 28)
#define BEAGLE_B200_FLAG_PARALLELOPS_GRID        (1L << 29)
#define BEAGLE_B200_FLAG_PREORDER_TRANSPOSE_MANUAL (1L << 30)
#define BEAGLE_B200_FLAG_PREORDER_TRANSPOSE_AUTO   (1L << 31)

/* Operation sizes and the "no buffer" index (BeagleOpCodes, beagle.h:201-205). */
#define BEAGLE_B200_OP_COUNT            7
#define BEAGLE_B200_PARTITION_OP_COUNT  9
#define BEAGLE_B200_OP_NONE             (-1)

/* Layout of BeagleOperation (beagle.h:870-878): seven ints per operation. */
typedef struct {
    int destinationPartials;
    int destinationScaleWrite;
    int destinationScaleRead;
    int child1Partials;
    int child1TransitionMatrix;
    int child2Partials;
    int child2TransitionMatrix;
} BeagleB200Operation;

/* Layout of BeagleOperationByPartition (beagle.h:922-932). */
typedef struct {
    int destinationPartials;
    int destinationScaleWrite;
    int destinationScaleRead;
    int child1Partials;
    int child1TransitionMatrix;
    int child2Partials;
    int child2TransitionMatrix;
    int partition;
    int cumulativeScaleIndex;
} BeagleB200OperationByPartition;

/* Layout of BeagleInstanceDetails (beagle.h:210-219). */
typedef struct {
    int resourceNumber;
    char* resourceName;
    char* implName;
    char* implDescription;
    long flags;
} BeagleB200InstanceDetails;

/* Layouts of BeagleResource / BeagleResourceList (beagle.h:224-237). */
typedef struct {
    char* name;
    char* description;
    long supportFlags;
    long requiredFlags;
} BeagleB200Resource;

typedef struct {
    BeagleB200Resource* list;
    int length;
} BeagleB200ResourceList;

/* ---- library / instance lifetime ------------------------------------- */
/* replaces beagleGetVersion (beagle.h:280) */
const char* beagleB200GetVersion(void);
/* replaces beagleGetResourceList (beagle.h:300): one resource per CUDA device,
 * in ordinal order; devices other than sm_100 carry no support flags */
BeagleB200ResourceList* beagleB200GetResourceList(void);
/* replaces beagleCreateInstance (beagle.h:378-391); resourceList[0], when
 * given, is the CUDA device ordinal.  Returns the instance index (>= 0). */
int beagleB200CreateInstance(int tipCount, int partialsBufferCount, int compactBufferCount,
                             int stateCount, int patternCount, int eigenBufferCount,
                             int matrixBufferCount, int categoryCount, int scaleBufferCount,
                             int* resourceList, int resourceCount, long preferenceFlags,
                             long requirementFlags, BeagleB200InstanceDetails* returnInfo);
/* replaces beagleFinalizeInstance (beagle.h:402) */
int beagleB200FinalizeInstance(int instance);
/* replaces beagleFinalize (beagle.h:412) */
int beagleB200Finalize(void);
/* replaces beagleSetCPUThreadCount (beagle.h:429-430); a GPU resource: returns
 * BEAGLE_B200_ERROR_NO_IMPLEMENTATION like the reference GPU implementation */
int beagleB200SetCPUThreadCount(int instance, int threadCount);

/* ---- data in / out ----------------------------------------------------- */
/* replaces beagleSetTipStates (beagle.h:446-448): patternCount states, >= stateCount = missing */
int beagleB200SetTipStates(int instance, int tipIndex, const int* inStates);
/* replaces beagleSetTipPartials (beagle.h:464-466): [pattern][state], copied to every category */
int beagleB200SetTipPartials(int instance, int tipIndex, const double* inPartials);
/* replaces beagleSetRootPrePartials (beagle.h:481-484): pre-order root = state frequencies */
int beagleB200SetRootPrePartials(int instance, const int* bufferIndices,
                                 const int* stateFrequenciesIndices, int count);
/* replaces beagleSetPartials (beagle.h:498-500): [category][pattern][state] */
int beagleB200SetPartials(int instance, int bufferIndex, const double* inPartials);
/* replaces beagleGetPartials (beagle.h:515-518) */
int beagleB200GetPartials(int instance, int bufferIndex, int scaleIndex, double* outPartials);
/* replaces beagleSetEigenDecomposition (beagle.h:534-538) */
int beagleB200SetEigenDecomposition(int instance, int eigenIndex, const double* inEigenVectors,
                                    const double* inInverseEigenVectors,
                                    const double* inEigenValues);
/* replaces beagleSetStateFrequencies (beagle.h:551-553) */
int beagleB200SetStateFrequencies(int instance, int stateFrequenciesIndex,
                                  const double* inStateFrequencies);
/* replaces beagleSetCategoryWeights (beagle.h:566-568) */
int beagleB200SetCategoryWeights(int instance, int categoryWeightsIndex,
                                 const double* inCategoryWeights);
/* replaces beagleSetCategoryRates (beagle.h:580-581) */
int beagleB200SetCategoryRates(int instance, const double* inCategoryRates);
/* replaces beagleSetCategoryRatesWithIndex (beagle.h:594-596) */
int beagleB200SetCategoryRatesWithIndex(int instance, int categoryRatesIndex,
                                        const double* inCategoryRates);
/* replaces beagleSetPatternWeights (beagle.h:608-609) */
int beagleB200SetPatternWeights(int instance, const double* inPatternWeights);
/* replaces beagleSetPatternPartitions (beagle.h:623-625) */
int beagleB200SetPatternPartitions(int instance, int partitionCount,
                                   const int* inPatternPartitions);

/* ---- transition matrices ----------------------------------------------- */
/* replaces beagleConvolveTransitionMatrices (beagle.h:661-665) */
int beagleB200ConvolveTransitionMatrices(int instance, const int* firstIndices,
                                         const int* secondIndices, const int* resultIndices,
                                         int matrixCount);
/* replaces beagleAddTransitionMatrices (beagle.h:681-685) */
int beagleB200AddTransitionMatrices(int instance, const int* firstIndices,
                                    const int* secondIndices, const int* resultIndices,
                                    int matrixCount);
/* replaces beagleTransposeTransitionMatrices (beagle.h:699-702) */
int beagleB200TransposeTransitionMatrices(int instance, const int* inputIndices,
                                          const int* resultIndices, int matrixCount);
/* replaces beagleUpdateTransitionMatrices (beagle.h:723-729): P(t) formed in FP64 */
int beagleB200UpdateTransitionMatrices(int instance, int eigenIndex,
                                       const int* probabilityIndices,
                                       const int* firstDerivativeIndices,
                                       const int* secondDerivativeIndices,
                                       const double* edgeLengths, int count);
/* replaces beagleUpdateTransitionMatricesWithModelCategories (beagle.h:753-759) */
int beagleB200UpdateTransitionMatricesWithModelCategories(int instance, int* eigenIndices,
                                                          const int* probabilityIndices,
                                                          const int* firstDerivativeIndices,
                                                          const int* secondDerivativeIndices,
                                                          const double* edgeLengths, int count);
/* replaces beagleUpdateTransitionMatricesWithMultipleModels (beagle.h:782-789) */
int beagleB200UpdateTransitionMatricesWithMultipleModels(int instance, const int* eigenIndices,
                                                         const int* categoryRateIndices,
                                                         const int* probabilityIndices,
                                                         const int* firstDerivativeIndices,
                                                         const int* secondDerivativeIndices,
                                                         const double* edgeLengths, int count);
/* replaces beagleSetTransitionMatrix (beagle.h:806-809) */
int beagleB200SetTransitionMatrix(int instance, int matrixIndex, const double* inMatrix,
                                  double paddedValue);
/* replaces beagleSetDifferentialMatrix (beagle.h:823-825) */
int beagleB200SetDifferentialMatrix(int instance, int matrixIndex, const double* inMatrix);
/* replaces beagleGetTransitionMatrix (beagle.h:840-842) */
int beagleB200GetTransitionMatrix(int instance, int matrixIndex, double* outMatrix);
/* replaces beagleSetTransitionMatrices (beagle.h:860-864) */
int beagleB200SetTransitionMatrices(int instance, const int* matrixIndices,
                                    const double* inMatrices, const double* paddedValues,
                                    int count);

/* ---- partials ------------------------------------------------------------ */
/* replaces beagleUpdatePartials (beagle.h:894-897): the whole operation list
 * runs as one op-walking kernel launch per call */
int beagleB200UpdatePartials(const int instance, const BeagleB200Operation* operations,
                             int operationCount, int cumulativeScaleIndex);
/* replaces beagleUpdatePrePartials (beagle.h:914-917) */
int beagleB200UpdatePrePartials(const int instance, const BeagleB200Operation* operations,
                                int operationCount, int cumulativeScaleIndex);
/* replaces beagleUpdatePartialsByPartition (beagle.h:947-949) */
int beagleB200UpdatePartialsByPartition(const int instance,
                                        const BeagleB200OperationByPartition* operations,
                                        int operationCount);
/* replaces beagleUpdatePrePartialsByPartition (beagle.h:964-966) */
int beagleB200UpdatePrePartialsByPartition(const int instance,
                                           const BeagleB200OperationByPartition* operations,
                                           int operationCount);
/* replaces beagleWaitForPartials (beagle.h:984-986) */
int beagleB200WaitForPartials(const int instance, const int* destinationPartials,
                              int destinationPartialsCount);

/* ---- scale factors -------------------------------------------------------- */
/* replaces beagleAccumulateScaleFactors (beagle.h:999-1002) */
int beagleB200AccumulateScaleFactors(int instance, const int* scaleIndices, int count,
                                     int cumulativeScaleIndex);
/* replaces beagleAccumulateScaleFactorsByPartition (beagle.h:1016-1020) */
int beagleB200AccumulateScaleFactorsByPartition(int instance, const int* scaleIndices, int count,
                                                int cumulativeScaleIndex, int partitionIndex);
/* replaces beagleRemoveScaleFactors (beagle.h:1033-1036) */
int beagleB200RemoveScaleFactors(int instance, const int* scaleIndices, int count,
                                 int cumulativeScaleIndex);
/* replaces beagleRemoveScaleFactorsByPartition (beagle.h:1052-1056) */
int beagleB200RemoveScaleFactorsByPartition(int instance, const int* scaleIndices, int count,
                                            int cumulativeScaleIndex, int partitionIndex);
/* replaces beagleResetScaleFactors (beagle.h:1067-1068) */
int beagleB200ResetScaleFactors(int instance, int cumulativeScaleIndex);
/* replaces beagleResetScaleFactorsByPartition (beagle.h:1080-1082) */
int beagleB200ResetScaleFactorsByPartition(int instance, int cumulativeScaleIndex,
                                           int partitionIndex);
/* replaces beagleCopyScaleFactors (beagle.h:1094-1096) */
int beagleB200CopyScaleFactors(int instance, int destScalingIndex, int srcScalingIndex);
/* replaces beagleGetScaleFactors (beagle.h:1107-1109) */
int beagleB200GetScaleFactors(int instance, int srcScalingIndex, double* outScaleFactors);

/* ---- likelihoods and derivatives ------------------------------------------ */
/* replaces beagleCalculateRootLogLikelihoods (beagle.h:1133-1139): FP64 site
 * sums and FP64 weighted reduction on the device */
int beagleB200CalculateRootLogLikelihoods(int instance, const int* bufferIndices,
                                          const int* categoryWeightsIndices,
                                          const int* stateFrequenciesIndices,
                                          const int* cumulativeScaleIndices, int count,
                                          double* outSumLogLikelihood);
/* replaces beagleCalculateRootLogLikelihoodsByPartition (beagle.h:1167-1176) */
int beagleB200CalculateRootLogLikelihoodsByPartition(int instance, const int* bufferIndices,
                                                     const int* categoryWeightsIndices,
                                                     const int* stateFrequenciesIndices,
                                                     const int* cumulativeScaleIndices,
                                                     const int* partitionIndices,
                                                     int partitionCount, int count,
                                                     double* outSumLogLikelihoodByPartition,
                                                     double* outSumLogLikelihood);
/* replaces beagleCalculateEdgeDerivatives (beagle.h:1218-1226): d lnL / d t for
 * every listed branch in one launch; per-site values, weighted sums and sums of squares */
int beagleB200CalculateEdgeDerivatives(int instance, const int* postBufferIndices,
                                       const int* preBufferIndices,
                                       const int* derivativeMatrixIndices,
                                       const int* categoryWeightsIndices, int count,
                                       double* outDerivatives, double* outSumDerivatives,
                                       double* outSumSquaredDerivatives);
/* Extension, no beagle.h counterpart: beagleUpdatePartials(operations, count,
 * BEAGLE_OP_NONE); then, when cumulativeScaleIndex is not BEAGLE_OP_NONE,
 * beagleResetScaleFactors(cumulativeScaleIndex) and
 * beagleAccumulateScaleFactors of every scale buffer the operations write;
 * then beagleCalculateRootLogLikelihoods(rootBufferIndex,
 * categoryWeightsIndex, stateFrequenciesIndex, cumulativeScaleIndex).  Same
 * results (to FP64 rounding of the sums) and error codes as those calls, and
 * the same ASYNCH delivery as beagleCalculateRootLogLikelihoods.  For 4-state
 * instances with 1, 2, 4 or 8 categories, at most 256 operations and the
 * root the last operation's destination, one kernel walks the list, keeps
 * each pattern's log scale factors in a register and forms the site
 * log-likelihood from the root row it has just written; other lists run as
 * the separate calls. */
int beagleB200UpdatePartialsWithRootLogLikelihood(int instance, const int* operations, int count,
                                                  int cumulativeScaleIndex, int rootBufferIndex,
                                                  int categoryWeightsIndex,
                                                  int stateFrequenciesIndex,
                                                  double* outSumLogLikelihood);
/* Extension, no beagle.h counterpart: beagleUpdatePrePartials(operations,
 * count, BEAGLE_OP_NONE) followed by beagleCalculateEdgeDerivatives over
 * (postBufferIndices[k], destination of operation k, derivativeMatrixIndices[k])
 * for k < count, sums only.  Same results and error codes as those two calls.
 * For 4-state instances with 1, 2, 4 or 8 categories, one kernel walks the
 * list (one launch per 256 operations) and forms each branch's derivative
 * from the pre-order row it has just computed (sibling pairs share their
 * loads); other shapes run the two calls. */
int beagleB200UpdatePrePartialsWithDerivatives(int instance, const int* operations, int count,
                                               const int* postBufferIndices,
                                               const int* derivativeMatrixIndices,
                                               const int* categoryWeightsIndices,
                                               double* outSumDerivatives,
                                               double* outSumSquaredDerivatives);
/* Extension, diagnostics: the kernel variant the autotuner last ran for this
 * instance, per kind: outVariants[0] post-order walk, [1] pre-order walk,
 * [2] edge derivatives, [3] fused pre-order + derivatives (0 = the two
 * calls' kernels, 1 = the fused walk).  -1 = default shape, -2 = not run. */
int beagleB200GetTunedVariants(int instance, int* outVariants);
/* replaces beagleCalculateCrossProductDerivative (beagle.h:1228-1236) */
int beagleB200CalculateCrossProductDerivative(int instance, const int* postBufferIndices,
                                              const int* preBufferIndices,
                                              const int* categoryRateIndices,
                                              const int* categoryWeightsIndices,
                                              const double* edgeLengths, int count,
                                              double* outSumDerivatives,
                                              double* outSumSquaredDerivatives);
/* replaces beagleCalculateEdgeLogLikelihoods (beagle.h:1265-1277) */
int beagleB200CalculateEdgeLogLikelihoods(int instance, const int* parentBufferIndices,
                                          const int* childBufferIndices,
                                          const int* probabilityIndices,
                                          const int* firstDerivativeIndices,
                                          const int* secondDerivativeIndices,
                                          const int* categoryWeightsIndices,
                                          const int* stateFrequenciesIndices,
                                          const int* cumulativeScaleIndices, int count,
                                          double* outSumLogLikelihood,
                                          double* outSumFirstDerivative,
                                          double* outSumSecondDerivative);
/* replaces beagleCalculateEdgeLogLikelihoodsByPartition (beagle.h:1314-1332): count 1;
 * lnL alone, or with both derivative sums (a first derivative alone returns
 * BEAGLE_B200_ERROR_NO_IMPLEMENTATION, as the reference CPU implementation does) */
int beagleB200CalculateEdgeLogLikelihoodsByPartition(
    int instance, const int* parentBufferIndices, const int* childBufferIndices,
    const int* probabilityIndices, const int* firstDerivativeIndices,
    const int* secondDerivativeIndices, const int* categoryWeightsIndices,
    const int* stateFrequenciesIndices, const int* cumulativeScaleIndices,
    const int* partitionIndices, int partitionCount, int count,
    double* outSumLogLikelihoodByPartition, double* outSumLogLikelihood,
    double* outSumFirstDerivativeByPartition, double* outSumFirstDerivative,
    double* outSumSecondDerivativeByPartition, double* outSumSecondDerivative);
/* replaces beagleGetLogLikelihood (beagle.h:1350-1351) */
int beagleB200GetLogLikelihood(int instance, double* outSumLogLikelihood);
/* replaces beagleGetDerivatives (beagle.h:1368-1370) */
int beagleB200GetDerivatives(int instance, double* outSumFirstDerivative,
                             double* outSumSecondDerivative);
/* replaces beagleGetSiteLogLikelihoods (beagle.h:1383-1384) */
int beagleB200GetSiteLogLikelihoods(int instance, double* outLogLikelihoods);
/* replaces beagleGetSiteDerivatives (beagle.h:1397-1399) */
int beagleB200GetSiteDerivatives(int instance, double* outFirstDerivatives,
                                 double* outSecondDerivatives);

/* ---- extensions (no counterpart in beagle.h) ---------------------------- */
/* The cudaStream_t (as void*) on which the instance queues all its work, for
 * callers that time it with CUDA events or order their own work against it.
 * The stream belongs to the instance and lives until it is finalised. */
int beagleB200GetCudaStream(int instance, void** outStream);

/* No counterpart in the reference (whose CUDA error path exits the process,
 * GPU/GPUInterfaceCUDA.cpp:98-104).  Every wait in this library's kernels (on
 * tensor-core completion or on bulk copies) is bounded; a wait that runs out
 * sets a device flag, the kernel finishes without its result, and the next
 * result call (getters, waitForPartials, synchronous calls) returns
 * BEAGLE_B200_ERROR_GENERAL, clears the flag and drops that evaluation's
 * pending results; the instance stays usable.  This call raises that flag on
 * the instance's stream as if a wait had run out (which = 0: tensor-core
 * kernels, 1: the bulk-copy derivative), so that a caller can exercise its
 * error path without a real time-out.  BEAGLE_B200_ERROR_OUT_OF_RANGE for
 * another `which` or while capturing. */
int beagleB200InjectKernelTimeout(int instance, int which);

/* No counterpart in the reference.  The pattern-weighted root log-likelihood
 * of caller-owned device buffers, for callers that cannot let a library call
 * cudaMalloc: frameworks that own all device memory through their own
 * allocator, or loops where cudaMalloc's implicit device synchronisation is not
 * acceptable.  The call allocates nothing.  Its only scratch, the per-block
 * partial sums of the FP64 reduction, is a fixed 64 KiB device array built into
 * the library (held on every GPU that loads it until the process exits), so
 * patternCount is limited to 8192 * 128 = 1,048,576; larger counts return
 * BEAGLE_B200_ERROR_OUT_OF_RANGE.
 *
 * All pointers except `stream` are device pointers on `device`:
 *   rootPartials            [patternCount][categoryCount][Sg], Sg = stateCount
 *                           rounded up to a multiple of 4 (this library's
 *                           partials layout); float if doublePrecision == 0,
 *                           else double; 16-byte aligned (rows are read as
 *                           16-byte vectors)
 *   categoryWeights         [categoryCount]     stateFrequencies  [stateCount]
 *   cumulativeScaleFactors  [patternCount] log scale factors, or NULL
 *   patternWeights          [patternCount]
 *   outSiteLogLikelihoods   [patternCount]      outSumLogLikelihood  [1]
 * The FP64 arrays must be 8-byte aligned.  A misaligned pointer returns
 * BEAGLE_B200_ERROR_OUT_OF_RANGE before anything is queued.
 * The work is queued on `stream` (a cudaStream_t; NULL = the default stream)
 * and the call returns without waiting.  Every call looks up the scratch
 * array's device address in the current context; the first call on a device
 * may load the library's device code to do so, so make that first call before
 * any stream capture.  Every call shares the array, so calls that overlap on the GPU race:
 * order them on one stream.  Calls from different host threads that target the
 * same device must not overlap either. */
int beagleB200RootLogLikelihoodsNoAlloc(int device, void* stream, const void* rootPartials,
                                        int doublePrecision, int stateCount, int patternCount,
                                        int categoryCount, const double* categoryWeights,
                                        const double* stateFrequencies,
                                        const double* cumulativeScaleFactors,
                                        const double* patternWeights,
                                        double* outSiteLogLikelihoods,
                                        double* outSumLogLikelihood);

/* ---- CUDA graphs of an instance's work (no beagle.h counterpart) ------
 * Between BeginCapture and EndCapture the calls on an ASYNCH instance
 * (BEAGLE_B200_FLAG_COMPUTATION_ASYNCH) are recorded into a CUDA graph instead
 * of running; LaunchGraph replays the recorded work on the instance's stream,
 * and the recorded result calls deliver again at the next synchronisation
 * point (getters, waitForPartials, synchronous calls), into the same caller
 * arrays, which must stay valid.  Calls that wait for results are refused with
 * BEAGLE_B200_ERROR_GENERAL while capturing.  Make the same calls once before
 * capturing so that every device table already has its size and contents;
 * argument tables that differ are copied through pinned memory the graph
 * keeps.  Typical use: capture partials, scaling, root lnL, pre-order partials
 * and edge derivatives once, then per step update the transition matrices
 * (outside the graph) and launch the graph; or capture the matrix update too
 * and launch with beagleB200LaunchGraphWithLengths.  Graphs live until the
 * instance is finalized. */
int beagleB200BeginCapture(int instance);
/* Returns the graph index in *graph. */
int beagleB200EndCapture(int instance, int* graph);
int beagleB200LaunchGraph(int instance, int graph);
/* The branch lengths of the transition-matrix updates captured in the graph
 * are read on the device when it runs.  This call replaces them (count = all
 * the captured updates' lengths, in capture order), then launches the graph,
 * so that a whole step -- P(t), partials, scaling, root lnL, pre-order
 * partials, derivatives -- is one call and one wait.  The lengths are copied
 * on the host (into pinned staging memory the graph owns) before the call
 * returns, so the caller may overwrite its array at once, pinned or not; they
 * stay: beagleB200LaunchGraph replays the lengths last given (the capture's
 * until this call replaces them).  Only the transition-matrix updates read
 * their lengths on the device: a captured beagleB200CalculateCrossProductDerivative
 * keeps the branch lengths it was captured with.
 * BEAGLE_B200_ERROR_OUT_OF_RANGE when count does not match the capture. */
int beagleB200LaunchGraphWithLengths(int instance, int graph, const double* lengths, int count);

/* ---- batches of instances (no beagle.h counterpart) ------------------
 * Many independent trees or partitions of uneven pattern and state counts,
 * one instance each, evaluated with a handful of launches per step instead of
 * one launch chain per instance.  A batch groups instances of one precision on
 * one device; while it exists they share one CUDA stream, so batch calls and
 * their single-instance calls stay ordered.  Per-member arguments are arrays
 * indexed by member position (the order of `instances` at creation); pointer
 * arrays hold one pointer per member.  Each member's arguments are validated
 * and mean what the single-instance call's arguments mean; an error in any
 * member returns its code before anything is queued for the rest of that
 * call's batched launches.
 *
 * Launches: transition matrices, one per (states, categories) group; post-
 * and pre-order walks and edge derivatives, one per category count for the
 * 4-state members (1, 2, 4 or 8 categories), the other members' own launches
 * otherwise; scale accumulation, root pre-partials, root log-likelihoods and
 * the final derivative sums, one each for all members. */
/* Returns the batch index (>= 0) or a negative code. */
int beagleB200CreateBatch(const int* instances, int count);
/* Members return to their own streams; the instances stay valid. */
int beagleB200FinalizeBatch(int batch);
/* beagleUpdateTransitionMatrices for every member: eigenIndices[m],
 * probabilityIndices[m][count[m]], edgeLengths[m][count[m]] (no derivative
 * matrices). */
int beagleB200BatchUpdateTransitionMatrices(int batch, const int* eigenIndices,
                                            const int* const* probabilityIndices,
                                            const double* const* edgeLengths,
                                            const int* counts);
/* beagleUpdatePartials for every member (7-int operations). */
int beagleB200BatchUpdatePartials(int batch, const int* const* operations,
                                  const int* operationCounts,
                                  const int* cumulativeScaleIndices);
/* beagleUpdatePrePartials for every member. */
int beagleB200BatchUpdatePrePartials(int batch, const int* const* operations,
                                     const int* operationCounts);
/* beagleAccumulateScaleFactors for every member, after zeroing its cumulative
 * buffer first when `reset` is nonzero (beagleResetScaleFactors). */
int beagleB200BatchAccumulateScaleFactors(int batch, const int* const* scaleIndices,
                                          const int* counts,
                                          const int* cumulativeScaleIndices, int reset);
/* beagleSetRootPrePartials for every member (one buffer each). */
int beagleB200BatchSetRootPrePartials(int batch, const int* bufferIndices,
                                      const int* stateFrequenciesIndices);
/* beagleCalculateRootLogLikelihoods for every member (one root each);
 * outSumLogLikelihoods[m].  Waits for the results, unless every member was
 * created with BEAGLE_B200_FLAG_COMPUTATION_ASYNCH: then the values are
 * written at beagleB200BatchWait, and the array must stay valid until then. */
int beagleB200BatchCalculateRootLogLikelihoods(int batch, const int* bufferIndices,
                                               const int* categoryWeightsIndices,
                                               const int* stateFrequenciesIndices,
                                               const int* cumulativeScaleIndices,
                                               double* outSumLogLikelihoods);
/* No beagle.h counterpart: beagleB200UpdatePartialsWithRootLogLikelihood for
 * every member (operations[i]: counts[i] 7-int post-order operations,
 * cumulativeScaleIndices[i] or BEAGLE_OP_NONE, rootBufferIndices[i],
 * categoryWeightsIndices[i], stateFrequenciesIndices[i]); lnL of member i in
 * outSumLogLikelihoods[i].  When every member is a 4-state instance with 1,
 * 2, 4 or 8 categories whose list ends at its root: one fused walk per
 * category count (each pattern's log scale factors summed in a register,
 * the site lnL formed from the root row); otherwise the batched calls of the
 * three steps.  Results delivered as beagleB200BatchCalculateRootLogLikelihoods
 * delivers them. */
int beagleB200BatchUpdatePartialsWithRootLogLikelihood(int batch, const int* const* operations,
                                                        const int* counts,
                                                        const int* cumulativeScaleIndices,
                                                        const int* rootBufferIndices,
                                                        const int* categoryWeightsIndices,
                                                        const int* stateFrequenciesIndices,
                                                        double* outSumLogLikelihoods);
/* beagleCalculateEdgeDerivatives for every member (sums only):
 * outSumDerivatives[m][counts[m]], outSumSquaredDerivatives[m][counts[m]]
 * (either may be NULL per member).  Waits for the results, or defers them to
 * beagleB200BatchWait as beagleB200BatchCalculateRootLogLikelihoods does. */
int beagleB200BatchCalculateEdgeDerivatives(int batch, const int* const* postBufferIndices,
                                            const int* const* preBufferIndices,
                                            const int* const* derivativeMatrixIndices,
                                            const int* categoryWeightsIndices,
                                            const int* counts,
                                            double* const* outSumDerivatives,
                                            double* const* outSumSquaredDerivatives);
/* No beagle.h counterpart: beagleB200UpdatePrePartialsWithDerivatives for
 * every member (operations[i]: counts[i] pre-order ops, postBufferIndices[i]
 * and derivativeMatrixIndices[i]: the node's post-order operand and
 * derivative matrix of each op's branch), sums in op order.  4-state members
 * with 1, 2, 4 or 8 categories run one batched fused walk per category
 * count; FP32 members with 4 < S <= 64 one batched tensor-core fused walk per
 * (S, C); other members their own call on the batch's stream.  Results as
 * beagleB200BatchCalculateEdgeDerivatives delivers them. */
int beagleB200BatchUpdatePrePartialsWithDerivatives(int batch, const int* const* operations,
                                                    const int* counts,
                                                    const int* const* postBufferIndices,
                                                    const int* const* derivativeMatrixIndices,
                                                    const int* categoryWeightsIndices,
                                                    double* const* outSumDerivatives,
                                                    double* const* outSumSquaredDerivatives);
/* Batch CUDA graphs (every member ASYNCH): the batch calls between
 * BeginCapture and EndCapture are recorded once as one graph of the batch's
 * stream (batched kernels, members' own launches, table uploads and result
 * copies); LaunchGraph replays it, and the captured calls' results reach the
 * caller's arrays at the next beagleB200BatchWait.  Run the sequence once
 * before capturing it.  Calls that wait for results are refused while
 * capturing. */
int beagleB200BatchBeginCapture(int batch);
int beagleB200BatchEndCapture(int batch, int* outGraph);
int beagleB200BatchLaunchGraph(int batch, int graph);
/* The branch lengths of the batch's transition-matrix updates captured in the
 * graph are read on the device when it runs.  This call replaces them, then
 * launches the graph, so that a whole batched step (matrices included) is
 * one call and one wait.  `lengths` holds all of them in capture order:
 * member by member in batch order, each member's lengths in the order its
 * captured calls listed them; count must match the capture
 * (BEAGLE_B200_ERROR_OUT_OF_RANGE otherwise).  They are copied on the host
 * before the call returns; beagleB200BatchLaunchGraph replays the lengths
 * last given. */
int beagleB200BatchLaunchGraphWithLengths(int batch, int graph, const double* lengths,
                                          int count);
/* Wait for everything queued on the batch's stream and write the deferred
 * results of ASYNCH members. */
int beagleB200BatchWait(int batch);

#ifdef __cplusplus
}
#endif
#endif /* BEAGLE_B200_H */
