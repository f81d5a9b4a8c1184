// Device layout of a batch of windows (host runtime <-> kernels).
//
// All windows of a solver are concatenated.  Per-window metadata lives in
// WinDesc; per-window LM state in WinLM (device-resident, updated by the
// kernels so that no host round trip is needed between LM iterations).
//
// Column spaces of window w:
//   retained  [0, Nr)   keyframe k: pose 15k..15k+5, speed/bias 15k+6..15k+14;
//                       then 6 per estimated extrinsic, then td.
//   visual    [0, Npc)  the columns a bearing factor can touch:
//                       pose k -> 6k, extrinsic e -> 6K+6e, td -> 6K+6E'.
//   landmark-local       keyframe slot j -> 6j (slot 0 = anchor keyframe), then
//                       one 6-column slot per extrinsic the landmark's observations
//                       touch (slot 0 = the anchor camera's), then td.
#pragma once
#include <cstdint>

namespace cgmli {

constexpr int kMaxTrackChunk = 32;     // factors per warp pass
constexpr int kMaxSupport = 64;        // keyframe slots per landmark
constexpr int kLinThreads = 256;       // linearization CTA
constexpr int kFactorThreads = 256;    // factorization CTA
// Reduced systems of at least kWideCols columns are factored by the wide
// sequence (several launches over the GPU) instead of one CTA per window.
constexpr int kWideCols = 288;
constexpr bool isWideWindow(int Nr) { return Nr >= kWideCols; }  // device code calls it too (relaxed constexpr)

struct WinDesc {
    int K, E, C, L, F, nImu;
    int Nr, Npc, ncalib;
    int estExt, estTd, hasTd;
    int kf0, ext0, cam0, lm0, obs0, imu0;
    int priorRank, priorCols, priorBlocks, priorBlk0;
    int vec0;            // offset of Nr-vectors (gret, dr, rhs)
    long long dense0;    // offset of Nr*Nr matrices (Hret, factor scratch)
    long long acc0;      // offset of the visual accumulator: Npc(Npc+1)/2 + 3*Npc
    long long sch0;      // offset of the Schur term: Npc(Npc+1)/2
    long long priorA0, priorR00, priorRef0;
    long long imuScratch0;  // nImu * 930 doubles (raw and whitened factor)
    long long priorScratch0;  // priorRank*priorCols + priorCols*6 doubles
    double huber, minInv;
    int charts;   // 1: some retained column is fixed or on the rotation-only chart (colChart)
    int fixedLm;  // 1: some landmark's inverse distance is held constant (lmFixed)
    // deterministic sums (cgmli_solver_options::deterministic): the window's slots in
    // DevBatch::detSlots, each Npc(Npc+1)/2 + Npc doubles (packed upper triangle, then a
    // vector): detPairs slots of J^T J and G_v, then detSchur slots of the Schur term and B_v
    long long det0;
    int detPairs, detSchur;
};
// Solve-time chart of a retained column (DevBatch::colChart).  A rotation-only
// extrinsic keeps its translation: its tangent theta maps to the full left
// SE(3) tangent as [rho; theta] = [[p]x; I] theta, so its rho columns are
// folded into its theta columns and then held like fixed columns.
enum { kColFree = 0, kColFixed = 1, kColRotTheta = 2, kColRotRho = 3 };

struct WinLM {
    double lambda, nu, cost, initialCost, linCost, trialCost, predicted, maxInc;
    int mode;        // kModeLinearize, kModeResolve, kModeDone
    int iterations, accepted, converged, status, acceptNow, trialValid;
    // outlier refits (a gated solve runs passes 0..R): iterations and accepted
    // steps at the start of the window's current pass, iterations charged to the
    // finished passes (at least one each), index of the window's current pass
    int passStart, passAccepted, charged, pass, pad;
    unsigned long long t0;  // device clock (ns) at the start of the solve, for the time budget
};
enum { kModeLinearize = 0, kModeResolve = 1, kModeDone = 2 };


// Pointers to every device array (filled by the host runtime).
struct DevBatch {
    int numWindows, numLandmarks, numObs, numKf, numExt, numCam, numImu, numRuns;
    int mixed;  // CGMLI_PRECISION_MIXED: FP32 Jacobians, weights and landmark sums in the linearization
    int minIterations;   // iterations before the time budget may end a window's solve
    long long budgetNs;  // time budget of a solve (0: none)
    const WinDesc* win;
    WinLM* lm;
    const int* bigFirst;  // windows by decreasing retained dimension: block order of the one-CTA-per-window
                          // kernels, so that the longest windows start first and the last wave is short
    // cameras
    const double* camR; const double* camT; const int* camExt;  // camExt: global extrinsic index
    // landmarks
    const int* lmWin; const int* lmKf; const int* lmCam; const int* lmObsBegin;  // lmObsBegin: numLandmarks+1
    const double* lmBearing; const double* lmVel; const double* lmTime;
    const int* lmNs; const int* lmNx; const int* lmSupp0; const int* supp;  // support: s keyframes (anchor first), then x extrinsics
    const long long* lmC0;                                // offset of the landmark's cross vector
    const unsigned short* lmUmap;  // per cross-vector entry: its column within the landmark's Schur chunk
    const int* schurCols;         // per Schur chunk: count, then the ascending visual columns
    double* lmC; double* lmD; double* lmG; double* lmCost; int* lmValid;
    double* lmDelta; double* lmPred; double* lmTrial; double* lmMaxInc; int* lmTrialValid;
    // observations
    const int* obKf; const int* obCam; const int* obSlot; const int* obXslot;
    const int* obLm;      // landmark (device index) of each observation
    const int* keyOrder;  // observations of each window sorted by (anchor kf, observer kf, anchor ext, observer ext)
    double* keyRows;      // weighted compact factor rows per observation (k_lin_landmark -> k_lin_pairs)
    const double* obBearing; const double* obP; const double* obVel; const double* obTime;
    // states: [0] accepted, [1] candidate
    double* pose[2]; double* sb[2]; double* ext[2]; double* td[2]; double* rho[2];
    double* rotKf[2]; double* rotExt[2];  // rotation matrices of the poses / extrinsics of each state (9 each)
    // IMU and priors
    const double* imu;  // numImu * sizeof(cgmli_frozen_imu)/8
    const int* imuKf;   // global keyframe index of the first state
    const signed char* colChart;     // per retained column (WinDesc::vec0 offsets): kCol*
    const unsigned char* lmFixed;    // per landmark: 1 = inverse distance held constant
    const int* priorKind; const int* priorIndex; const int* priorCol; const int* priorOff;  // per prior block
    const double* priorA; const double* priorR0; const double* priorRef;
    // per-window dense storage
    double* Hret; double* gret; double* costRet; double* trialRet; int* retValid;
    double* acc;     // visual accumulators: J^T J (packed upper), unused, G_v, B_v
    double* sch;     // Schur term sum_l c_l c_l^T / dt_l (packed upper)
    double* dr;      // state increments (Nr per window)
    double* rhs;
    double* Sglob;   // damped reduced system and its Cholesky factor (Nr x Nr column-major, lower)
    double* imuScratch; double* priorScratch;
    double* predState;
    int* solveStatus;
    // wide windows (isWideWindow): their indices, x / undamped diagonal / damping
    // (3 Nr per window at 3 vec0) and a factorization-failed flag per window
    const int* wideList;
    double* facVec;
    int* facFailed;
    // per wide window (at its wideList position times (ceil(wideCols / 32) + 1) wideCols):
    // the row parts of the undamped product by 32-column block, then its column parts
    double* wideProd;
    // per wide window, two panel buffers (by panel parity) of 32 x wideCols: a panel's
    // solved L21 (k-major) until it is stored into Sglob
    double* wideL21;
    double* detSlots;  // deterministic mode: per-unit partial sums (WinDesc::det0)
    double* out;     // per-window scratch for read-back (costs)
};

// ---- marginalization (one victim keyframe per window) ----------------------------
// Column space of window w: victim pose and speed/bias [0, nm), then the
// separator [nm, m) in block order (keyframes ascending with pose before
// speed/bias, then extrinsics, then td).  H holds the upper triangle
// (row <= column) of the m x m information, row-major.
constexpr int kMargMaxNc = 200;     // marginalization columns touched by one eliminated landmark
constexpr int kMargMaxSep = 1024;   // separator columns (Jacobi pair tables hold 512 pairs)
constexpr int kPriorMaxCols = kMargMaxSep;  // tangent columns of a window's prior (what a marginalization forms)
constexpr int kMargThreads = 512;   // victim CTAs
constexpr int kEigenThreads = 512;  // eigen CTAs
// Schur chunks of the linearization (k_lin_schur): rows x padded width of the
// chunk's column union + 1 fit the CTA's shared rows.
constexpr int kSchurThreads = 256;
constexpr int kSchurSmemDoubles = 8192;
constexpr int kSchurMaxRows = 128;
// Deterministic mode: a window's pair chunks and its Schur chunks are split into
// contiguous units, each summed into a slot of its own: about kDetUnitObs key-ordered
// observations per pair unit and kDetSchurChunksPerUnit Schur chunks per Schur unit
// (enough units to fill the GPU without a tail of long units from the largest windows),
// at most kDetMaxSlots units of each kind per window (the slots' memory).
constexpr int kDetMaxSlots = 128;
constexpr int kDetUnitObs = 256;
constexpr int kDetSchurChunksPerUnit = 2;
inline bool schurChunkFits(int rows, int unionCols) {
    const int np = (unionCols + 1 + 31) / 32 * 32;
    return rows <= kSchurMaxRows && (long long)rows * np <= kSchurSmemDoubles;
}
constexpr int kMargLmThreads = 128; // one CTA per eliminated landmark (windows above kRowsMaxN)
constexpr int kRowsMaxN = 256;      // visual columns of a window on the dense-row path
constexpr int kRowsCap = 96;        // rows of one dense-row chunk (2 per observation + 1 per landmark)
constexpr int kRowsThreads = 512;   // dense-row CTAs
constexpr int kMargRecord = 56;     // staged doubles per observation of an eliminated landmark

struct MargWin {
    int m, nm, nr;          // m = 0: window not marginalized
    int elim0, nElim;       // eliminated landmarks in MargBatch::elim
    int imu[2];             // consumed IMU factors (global index) or -1
    int tdCol;              // column of td or -1
    int hasPrior;           // the window carries a prior
    long long H0;           // m * m
    long long sep0;         // nr * nr: separator information, eigenvectors, A
    long long vec0;         // m
    long long x0;           // 2 * 15 * (nr + 1): victim solve scratch, then the fast path's vectors
    double huber;
    int nv;                 // visual columns (poses, extrinsics, td) in column order
    int vis0;               // offset of the window's visual -> marginalization column map
    int visTd;              // visual column of td or -1
    int rowsPath;           // 1: eliminated landmarks accumulate through dense rows (nv <= kRowsMaxN)
    int imuAll;             // 1: every IMU factor of the window is consumed (calibration information)
};
struct MargElim { int lm, win, nc, col0, obs0; };  // device landmark, window, local columns, offsets
struct MargBatch {
    int numWindows, numElim;
    long long eigenSmem;  // dynamic shared memory of the eigen CTA (packed separator, eigenvectors when they fit)
    long long fastSmem;   // dynamic shared memory of the full-rank fast path
    long long triSmem;    // dynamic shared memory of the tridiagonal eigen path
    const MargWin* win;
    const int* bigFirst;  // windows by decreasing width of their larger block: block order of the
                          // one-CTA-per-window kernels
    const MargElim* elim;
    const int* cols;     // local column -> marginalization column
    const int* obsMap;   // 5 per observation of an eliminated landmark: local start of
                         // anchor pose, observer pose, anchor extrinsic, observer extrinsic, td (-1 if none)
    const int* poseCol; const int* sbCol; const int* extCol;  // global keyframe / extrinsic -> column or -1
    double* H; double* b; double* sepH; double* sepV; double* sepB; double* evals; double* A; double* r0; double* X;
    double* maxD;        // per window: largest eliminated landmark information
    double* stats;       // 4 per window: robust cost, whitened |r|^2, eliminated reduction, cutoff
    int* rank; int* status;
    int* fast;           // per window: 1 when the fast path formed the prior, 3 the tridiagonal eigen path, 0 neither;
                         // 2 while the fast path's saved tridiagonal form waits for the eigen path
    // dense-row path
    double* rows;        // kMargRecord per eliminated observation (staged factor rows)
    const int* visCol;   // visual column -> marginalization column, per window from MargWin::vis0
    const int* visPose; const int* visExt;  // global keyframe / extrinsic -> visual column or -1
    const int4* chunks;  // {first, end eliminated landmark, first, end staged observation}: <= kRowsCap rows
    const int4* items;   // {window, first chunk, end chunk, -}: one CTA each
    int numItems;
    long long rowsSmem;  // dynamic shared memory of a dense-row CTA
    const int* slowElim; // eliminated landmarks of windows above kRowsMaxN (one CTA each)
    int numSlowElim;
};

// Parts of one LM iteration's launch sequence (launchIterationParts).
enum { kIterLinearize = 1, kIterStep = 2, kIterDecide = 4 };

// Called before (phase 0) and after (phase 1) every kernel launch of an
// iteration; used for per-kernel event timing.
typedef void (*LaunchHook)(void* ctx, int kind, int phase);

// Per-window counters of the NIS gate: evaluated by the last gate, rejected by
// the last gate after a solve, rejected in total, a residual was not finite,
// rejected by the gate before the first solve; one spare.
constexpr int kGateCounts = 6;

// Kernel shapes the autotuner chooses between: warps per CTA and the CTAs per SM
// the register budget is compiled for (launch bounds), for the landmark pass
// (k_lin_landmark) and the trial pass (k_trial).  More CTAs per SM cap the
// registers lower (168 at 12 warps per SM, where the FP64 factor chain spills);
// one CTA per SM lets a thread keep its chain in up to 255 registers.
struct KernelShape { int warps, minBlocks; };
constexpr int kLinShapes = 4;
constexpr KernelShape kLinShapeTable[kLinShapes] = {{6, 2}, {8, 1}, {4, 3}, {6, 1}};
constexpr int kTrialShapes = 3;
constexpr KernelShape kTrialShapeTable[kTrialShapes] = {{8, 2}, {8, 1}, {4, 4}};

// Work decomposition of one batch (device pointers and counts).
struct LaunchPlan {
    const int4* runs;        // {window, first tile, end tile, -}: one warp each (landmark order)
    const int2* tiles;       // {first landmark, end landmark}, <= 32 observations
    int numTiles;
    const int4* pairChunks;  // {window, first key-ordered index, end, -}: <= 32 observations, one warp each
    int numPairChunks;
    const int4* schurChunks; // {window, first landmark, end landmark, -}: one CTA each
    int numSchurChunks;
    int maxNs;               // widest landmark support of the batch (local columns)
    size_t facSmem;          // k_factor (windows below kWideCols)
    int linShape, trialShape;  // kLinShapeTable / kTrialShapeTable entries
    int numWide;             // wide windows (B.wideList)
    int wideCols;            // largest wide Nr: panels and trailing tiles of the sequence
    int wideCharts;          // some wide window has solve-time charts
    size_t wideFinishSmem;
    // deterministic mode (WinDesc::det0): pair units {window, first key-ordered position,
    // end, slot} (one warp each) and Schur units {first Schur chunk, end chunk, slot,
    // window} (one CTA each); 0 units: the atomic form
    const int4* detPairs;
    int numDetPairs;
    const int4* detSchur;
    int numDetSchur;
};

}  // namespace cgmli
