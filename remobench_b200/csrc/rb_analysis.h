// Analysis stage types shared by rb_analysis.cu and the host orchestration.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "rb_kernels.h"
#include "rb_state.h"

namespace rb {

// Exact sums of a node's subtree in the node's own frame: n, S1 = Σq (u64),
// S2 = Σqqᵀ (xx xy xz yy yz zz as lo/hi u64 pairs), newest batch that touched it.
struct RollSum {
    unsigned long long n;
    unsigned long long s1[3];
    unsigned long long s2[12];
    unsigned long long c1[3];  // Σ of the 8-bit r, g, b
    unsigned long long c2[3];  // Σ of their squares
    uint32_t lastTouched;
    uint32_t pad;
};

constexpr int kNumFeatures = 16;

// How Refinement ranks the frontier (rb_analysis_params.score_mode).
enum ScoreMode : uint32_t {
    kScorePartial = 0,     // current (partial) surface variation x coverage
    kScoreClosed = 1,      // closure-lagged: closed nodes only, open nodes score 0
    kScoreLearned = 2,     // closed: their surface variation; open: the MLP's prediction
};

enum AnalysisFlags : uint32_t {
    kAnalysisFp64 = 1u,      // the eigen-solve took the FP64 branch
    kAnalysisLarge = 2u,     // projected extent above the pixel budget
    kAnalysisFrontier = 4u,  // inner, not large, parent large: drawn as one item now
};

struct NodeAnalysis {
    float eig[3];            // descending, units of (node size)^2
    float normal[3];         // eigenvector of eig[2]
    float surfaceVariation;  // eig[2] / (eig[0] + eig[1] + eig[2])
    float planarity;         // (eig[1] - eig[2]) / eig[0]
    float coverage;          // fraction of the frame covered by the node's projected box
    float score;             // geometric score x coverage
    unsigned long long count;
    uint32_t lastTouched;
    uint32_t closed;
    uint32_t flags;
    uint32_t pad;
};

struct AnalysisParams {
    uint32_t minPoints;      // nodes with fewer points score 0
    uint32_t closureMargin;  // batches without new points before a node counts as closed
    uint32_t currentBatch;
    uint32_t frontierOnly;   // queue only nodes Refinement can open (kAnalysisFrontier)
    float pixelBudget;
    uint32_t scoreMode;      // ScoreMode
};

struct AnalysisCounters {
    uint32_t fp64Branch;
    uint32_t eligible;
    uint32_t thresholdBin;
    uint32_t numCandidates;
    uint32_t queueLength;
    uint32_t overflow;
    uint32_t pad[2];
};

void launchRollLevel(const Dev& d, RollSum* roll, uint32_t level, int grid, cudaStream_t s);
void launchAnalyze(const Dev& d, const RollSum* roll, NodeAnalysis* out, float* features,
                   const AnalysisParams& p, const Frame& f, AnalysisCounters* ac, int grid, cudaStream_t s);
// Score and queue key per node; predictions (2 per node) are read in kScoreLearned mode.
void launchScore(const Dev& d, NodeAnalysis* out, const float* predictions, unsigned long long* keys,
                 const AnalysisParams& p, AnalysisCounters* ac, int grid, cudaStream_t s);
void launchQueue(const Dev& d, const unsigned long long* keys, uint32_t* hist, unsigned long long* cand,
                 uint32_t candCap, uint32_t K, uint32_t* queue, AnalysisCounters* ac, int grid, cudaStream_t s);
void launchRefineMask(const Dev& d, const uint32_t* queue, const AnalysisCounters* ac, uint32_t budget,
                      uint8_t* mask, int grid, cudaStream_t s);
cudaError_t configureQueueSort(uint32_t candCap);

}  // namespace rb
