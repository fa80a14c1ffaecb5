// The device half of a world: SoA arenas in HBM, per-step scratch, and the
// launchers of every stage of the step.  Host code (world.cu) owns one
// DevWorld per m3d_world and drives the stages in the reference's order.
#pragma once

#include "m3d_types.cuh"
#include "prims.cuh"

namespace m3d_diff
{
struct TapeContact;
}

namespace m3g
{

// Counters written by the kernels and read back by the host at the few
// points where the step needs a size (pinned host copy, one D2H each).
struct StepCounters
{
	uint32_t activeEntries;
	uint32_t stableEntries;
	uint32_t activeOversized;
	uint32_t stableOversized;
	uint32_t runs;
	uint32_t gridPairs;
	uint32_t overPairs;
	uint32_t newContacts;
	uint32_t removed;
	uint32_t endRemoval;
	uint32_t beginNP;
	uint32_t endNP;
	uint32_t anyAwakeDynamic;
	uint32_t islandCount;
	uint32_t touchingCount;
	uint32_t awakeIslands;
	uint32_t islandContacts;
	uint32_t islandJoints;
	uint32_t islandBodies;
	uint32_t stableDirty;
	uint32_t bodyCount;
	uint32_t awakeBodyCount;
	uint32_t hashFail;
	uint32_t coloredIslands;
	uint32_t serialIslands;
	uint32_t freeIslands;
	uint32_t waitErrors; // bounded device waits that ran out (non-zero: results of the step are suspect)
	uint32_t contactCount; // live contacts (device-side count during the step)
	uint32_t giantIslands; // islands solved by the whole-GPU coloured kernel
	uint32_t keptStable;     // batch: stable entries of worlds that keep their tier
	uint32_t keptStableOver; // batch: their oversized bodies
	uint32_t keptContacts;   // batch: contacts after the world-major re-layout
	uint32_t tinyIslands;    // serial islands small enough for one thread each
	uint32_t warpIslands;    // the other serial islands (one warp each)
	uint32_t islandPoints;   // manifold points of the island contacts (before the solve)
	uint32_t serialBodies;   // bodies of the serial islands
	uint32_t serialContacts; // contacts of the serial islands
	uint32_t sleptBodies;    // bodies put to sleep (counted only while a tape records)
	uint32_t tinyBodies;     // bodies of the tiny serial islands (one thread each)
	uint32_t tinyContacts;   // contacts of the tiny serial islands
};

// Host -> device body update record (one per body touched by the API
// between two steps).
enum UploadMask : uint32_t
{
	kUpAll = 1u << 0,       // freshly created body: every field
	kUpPose = 1u << 1,      // position + rotation
	kUpVel = 1u << 2,       // linear + angular velocity
	kUpIW = 1u << 3,        // world inverse inertia
	kUpForce = 1u << 4,     // force + torque
	kUpState = 1u << 5,     // inUse / awake / enableSleep / sensor + sleep timers
	kUpCold = 1u << 6,      // materials (also refreshes live contacts)
	kUpFatReset = 1u << 7,  // fat AABB invalid (teleport / recycled slot)
};

struct BodyUpload
{
	int32_t index;
	uint32_t mask;
	float4 pos, rot, vel, angVel;
	float4 massInv;
	float4 iw0, iw1, iw2;
	float4 force, torque;
	float2 sleep;
	uint32_t state;
	BodyCold cold;
};

// Island table entry.  Ranges index the label-sorted body / contact / joint
// lists of the step.
struct IslandRec
{
	int32_t bodyStart, bodyCount;
	int32_t contactStart, contactCount;
	int32_t jointStart, jointCount;
	int32_t label;
	int32_t kind; // 0 free bodies, 1 serial Gauss-Seidel, 2 graph coloured (one CTA), 3 giant (whole GPU)
};

struct DevWorld
{
	cudaStream_t stream = nullptr;
	PrimScratch prim;

	BodySoA B = {};
	ContactSoA C = {};
	int32_t bodyCap = 0;
	int32_t contactCap = 0;
	int32_t contactCount = 0;

	// joints (mirror of the host table) and the sorted jointed-pair keys
	DevBuf joints;
	int32_t jointCount = 0;
	DevBuf jointedPairs;
	int32_t jointedCount = 0;

	// per-body step scratch
	DevBuf inActiveCells, inStableCells; // u8
	DevBuf cellCountA, cellCountS;       // u32
	DevBuf overFlagA, overFlagS;         // u32
	DevBuf label;                        // i32 union-find parent / island label
	DevBuf islandFlag;                   // u32 per label: awake
	DevBuf colorMask;                    // u32
	DevBuf matDirty;                     // u8
	DevBuf sleepFirstNo, sleepMin;       // per label
	DevBuf bodyKeys, bodyVals;           // label-sorted island bodies

	// grid (active tier rebuilt every step, stable tier on demand)
	DevBuf activeKeys, activeVals, stableKeys, stableVals;
	DevBuf activeOver, stableOver;
	int64_t activeEntries = 0, stableEntries = 0;
	int32_t activeOverCount = 0, stableOverCount = 0;
	DevBuf runStarts, runFlag, runOffs;
	int32_t runCount = 0; // upper bound of the cell runs (exact count on the device)
	DevBuf entryOffsA, entryOffsS, overOffsA, overOffsS;
	DevBuf keyRanges;               // per tier: min x, y, z then max x, y, z of the key fields (u32)
	uint32_t* hostRanges = nullptr; // pinned copy, 12 words

	// pair build
	DevBuf runPairCount, runPairOffs; // u32 per run
	DevBuf overKeys;              // u64 per oversized candidate
	DevBuf keepScan;
	int64_t pairTotal = 0;        // admitted pairs (upper bound of new contacts)
	int32_t contactMax = 0;       // upper bound of the device contact count
	DevBuf pairKeys;              // u64 admitted candidates in emission order
	DevBuf overFlag, overScan;    // oversized candidate flags
	int64_t overTotal = 0;        // length of the oversized candidate stream
	DevBuf existingSet;           // hash set of existing contact keys
	uint32_t existingMask = 0;
	DevBuf newSet, newSetPos;     // first-occurrence dedupe
	uint32_t newMask = 0;
	DevBuf keepFlag;              // u32 per admitted candidate
	DevBuf newContactKeys;

	// removal / narrowphase / events
	DevBuf removeFlag, removeScan; // u32 per contact
	DevBuf moveSrc;                // i32 per hole rank
	DevBuf adjCount, adjStart;     // u32 per body + 1: contacts touching each body (CSR)
	DevBuf adjList;                // i32, 2 per contact
	DevBuf transition;             // i8 per contact
	DevBuf evBeginFlag, evEndFlag; // u32 per contact
	DevBuf evBegin, evEnd;         // int4 (bodyA, bodyB, sensor, 0)
	DevBuf evRemoval;              // int4, descending contact index

	// islands
	DevBuf contactKeys, contactVals; // label-sorted island contacts
	DevBuf jointKeys, jointVals;
	DevBuf islandStartFlag, islands; // IslandRec
	DevBuf islandKinds;
	DevBuf labelCount, labelStart, labelCursor; // per label: island bodies
	DevBuf islandListFlag, islandListOffs, islandLabels, coloredList, serialList, tinyList, giantList, jointScan;
	DevBuf tinyKeys; // sort keys of the tiny-island list
	int32_t islandMax = 0; // upper bound of the awake islands of the step
	uint32_t lastSerialIslands = 0; // serial islands of the previous step (kernel choice)
	// serial islands of at most tinyContacts contacts (no joints) take one
	// thread each when the previous step had more than tinyModeIslands serial
	// islands (m3d_gpu_autotune may change both; results do not depend on them)
	int32_t tinyContacts = kTinyIslandContacts;
	uint32_t tinyModeIslands = kTinyModeIslands;
	int32_t islandCount = 0;
	int32_t islandsBuiltFor = 0; // body count of the last island build (0: never)
	DevBuf colorOf;      // per island-contact position: colour 0..8
	DevBuf colorOrder;   // island contacts regrouped by colour
	DevBuf colorStart;   // per island: 10 offsets into colorOrder
	DevBuf packetMax;    // per colorOrder position: max points of its packet
	DevBuf contactColor; // per contact: colour for introspection

	// giant islands (k_giant.cu): coloured across the whole GPU
	int32_t giantIslandContacts = 32768; // islands with at least this many contacts
	DevBuf giantLocal, giantBodyOffs, giantBodyCursor, giantIncidence, giantPred, giantDone, giantChunkHist;
	DevBuf giantMisc, giantBarrier;
	DevBuf giantOvOrder, giantLevelStart; // overflow bucket regrouped by level, level offsets
	uint32_t giantEpoch = 0;
	int giantGrid = 0;

	DevBuf uploads;      // BodyUpload staging (device)
	DevBuf counters;     // StepCounters
	StepCounters* hostCounters = nullptr; // pinned

	DevBuf queryOut;     // query results

	// batch of worlds packed into this arena (m3d_gpu_batch_create): bodies of
	// world w are contiguous, cell keys carry the world above the cell
	// coordinates, contacts are kept world-major (each world's contacts in its
	// own reference order) and the stable tier is rebuilt per world
	bool batched = false;
	int32_t worldCount = 1;
	int keyBits = 21;            // bits per cell coordinate in a cell key
	DevBuf worldOf;              // u32 per body (B.world)
	DevBuf worldFirstBody;       // u32 per world + 1: first body slot of each world
	int32_t maxWorldBodies = 0;  // largest world (body slots)
	DevBuf overBlockOffs;        // oversized candidate blocks, world by world
	DevBuf overBlockCount;       // their sizes (scanned into overBlockOffs)
	DevBuf worldRebuild;         // u8 per world: stable tier rebuilt this step
	DevBuf worldStableDirty;     // u32 per world: stable tier made dirty on the device
	DevBuf worldContactCount;    // u32 per world: contacts at the start of the step
	DevBuf worldContactStart;    // u32 per world + 1
	DevBuf worldNewCount, worldNewStart, worldVStart, worldRemoved, worldFinalStart; // u32 per world + 1
	DevBuf newByWorldKeys, newByWorldVals; // new contacts grouped by world (emission order inside)
	DevBuf vFlag, vScan, vSrc;   // per virtual contact (old then new, world-major)
	DevBuf keptKeys, keptVals, keptOver; // stable-tier entries of worlds that keep their tier
	ContactSoA C2 = {};          // second contact arena: target of the world-major re-layout

	// differentiation tape (k_diff.cu): set for a step that records
	bool recording = false;
	m3d_diff::TapeContact* tapeContacts = nullptr; // this step's contact records
	uint32_t* sleepRecord = nullptr;               // bodies put to sleep this step
	DevBuf tapeGen;                                // per contact: what this step's narrowphase did to its manifold
};

// one stable-dirty word per world (StepCounters::stableDirty for one world)
uint32_t* stableDirtyWords(DevWorld& w);

// ---- launchers (defined in k_*.cu) -----------------------------------------

bool growBodies(DevWorld& w, int32_t capacity);
bool growContacts(DevWorld& w, int32_t capacity);
void readCounters(DevWorld& w); // stream sync + D2H of StepCounters
void setDeviceCount(DevWorld& w, uint32_t* p, uint32_t v); // stream-ordered store
void resetStepCounters(DevWorld& w, uint32_t contactCount); // StepCounters zero but contactCount, one launch
StepCounters* devCounters(DevWorld& w);

void launchApplyUploads(DevWorld& w, const BodyUpload* hostRecs, int32_t count);
void launchMaterialRefresh(DevWorld& w);

// broadphase (k_broadphase.cu); the step's host syncs sit between
// launchEmitGrid / launchSortGrid and launchPairCount / launchPairEmit
void launchRefresh(DevWorld& w, int32_t n, float dt, bool rebuildStable, float cellSize);
void launchEmitGrid(DevWorld& w, int32_t n, float cellSize, bool rebuildStable);
void launchSortGrid(DevWorld& w, bool rebuildStable);
void launchFindRuns(DevWorld& w);
void launchPairCount(DevWorld& w, int32_t n, float cellSize);
void launchPairEmit(DevWorld& w, int32_t n, float cellSize);
void launchCreateContacts(DevWorld& w);
void launchRemoval(DevWorld& w);
// destroy-time swap-removes computed on the host: move (dst, src) pairs
void launchContactMoves(DevWorld& w, const int2* hostMoves, int32_t count);
void launchContactAdjacency(DevWorld& w, int32_t bodies, cudaStream_t s, PrimScratch& prim);

// batch of worlds (k_batch.cu)
void launchKeepStable(DevWorld& w, uint32_t* ranges);
void launchAppendKeptStable(DevWorld& w, int64_t fresh, int32_t freshOver);
void launchBatchRelayout(DevWorld& w);

// narrowphase (k_narrow.cu)
void launchNarrowphase(DevWorld& w, float dt);

// islands, sleep, kinematics (k_islands.cu)
void launchAnyAwakeDynamic(DevWorld& w, int32_t n);
void launchIslands(DevWorld& w, int32_t n);
void launchSleep(DevWorld& w, float dt);
void launchFinish(DevWorld& w, int32_t n, float dt, bool clearForces);

// solver (k_solve.cu, k_giant.cu)
struct SolveParams;
void launchSolve(DevWorld& w, float dt, int substeps, V3 gravity, int positionIterations);
void launchSolveGiant(DevWorld& w, const SolveParams& P);

// queries (k_query.cu)
struct RayQueryOut
{
	int32_t body;
	float fraction;
	float point[3];
	float normal[3];
	int32_t hit;
};
void launchRayCast(DevWorld& w, int32_t n, V3 origin, V3 translation, uint32_t maskBits, float cellSize,
				   RayQueryOut* hostOut);
void launchSphereCast(DevWorld& w, int32_t n, V3 origin, float radius, V3 translation, uint32_t maskBits,
					  RayQueryOut* hostOut);
void launchOverlap(DevWorld& w, int32_t n, Box box, uint8_t* hostFlags);

// sphere cast into a caller-provided device scratch block of
// sphereCastScratchBytes(n) bytes, 16-byte aligned
constexpr size_t kCastRecBytes = 28;
size_t sphereCastScratchBytes(int32_t n);
void launchSphereCastInto(DevWorld& w, int32_t n, V3 origin, float radius, V3 translation, uint32_t maskBits,
						  void* scratch, RayQueryOut* hostOut);

// differentiation tape (k_diff.cu); status returns are M3D_GPU_* codes
struct DiffTape;
DiffTape* tapeCreate(DevWorld& w, int32_t nBodies, int checkpointEvery);
void tapeDestroy(DiffTape* t);
void tapeMarkUnsupported(DiffTape* t, const char* why);
const char* tapeUnsupported(const DiffTape* t); // null while the tape is differentiable
int32_t tapeSteps(const DiffTape* t);
int64_t tapeBytes(const DiffTape* t); // device bytes of the recorded steps (records, tables, checkpoints)
int64_t tapeWarpIslands(const DiffTape* t); // islands of the recorded steps worked by a warp each
void tapeStepBegin(DiffTape* t, DevWorld& w, int32_t n, float dt, int substeps, V3 g, int iterations);
void tapeBeforeIslands(DiffTape* t, DevWorld& w, int substeps);
void tapeStepEnd(DiffTape* t, DevWorld& w, const StepCounters& hc);
int32_t tapeReplay(DiffTape* t, DevWorld& w, float* pos, float* rot, float* vel, float* angVel, int32_t capacity);
int32_t tapeBackward(DiffTape* t, DevWorld& w, const float* dPos, const float* dRot, const float* dVel,
					 const float* dAngVel, float* gPos, float* gRot, float* gVel, float* gAngVel, float* gMass,
					 float* gFriction, float* gRestitution, int32_t capacity);
int32_t tapeBackwardHost(DiffTape* t, const double* dPos, const double* dRot, const double* dVel,
						 const double* dAngVel, double* gPos, double* gRot, double* gVel, double* gAngVel,
						 double* gMass, double* gFriction, double* gRestitution, int32_t capacity);
int32_t tapeRegenerateHost(DiffTape* t, int doublePrecision, const double* dVel, const double* dAngVel,
						   const double* dMass, const double* dFriction, const double* dRestitution, double* pos,
						   double* rot, double* vel, double* angVel, int32_t capacity);

} // namespace m3g
