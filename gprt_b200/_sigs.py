"""ctypes signatures of every symbol include/gprtcu.h and include/gprt_compat.h declare."""
import ctypes

vp = ctypes.c_void_p
u32 = ctypes.c_uint32
u64 = ctypes.c_uint64
i64 = ctypes.c_int64
sz = ctypes.c_size_t
i32 = ctypes.c_int
st = ctypes.c_int  # gprtcuStatus

SIGNATURES = {
    "gprtcuStatusString": ([i32], ctypes.c_char_p),
    "gprtcuVersion": ([], i32),
    "gprtcuScratchStatus": ([vp, vp, ctypes.POINTER(i32)], st),
    "gprtcuScanScratchSize": ([u64], sz),
    "gprtcuExclusiveSumU32": ([vp, vp, u64, vp, vp, sz, vp], st),
    "gprtcuInclusiveSumU32": ([vp, vp, u64, vp, vp, sz, vp], st),
    "gprtcuExclusiveSumU32NoAlloc": ([vp, vp, u64, vp, vp], st),
    "gprtcuPartitionI32": ([vp, vp, u64, i32, vp, vp, sz, vp], st),
    "gprtcuSelectI32": ([vp, vp, u64, i32, vp, vp, sz, vp], st),
    "gprtcuSortScratchSize": ([u64, i32, i32], sz),
    "gprtcuSortKeysU32": ([vp, u64, i32, i32, vp, sz, vp], st),
    "gprtcuSortPairsU32": ([vp, vp, u64, i32, i32, vp, sz, vp], st),
    "gprtcuSortKeysU64": ([vp, u64, i32, i32, vp, sz, vp], st),
    "gprtcuSortPairsU64": ([vp, vp, u64, i32, i32, vp, sz, vp], st),
    "gprtcuSortPairsU32U64": ([vp, vp, u64, i32, i32, vp, sz, vp], st),
    "gprtcuSortPairsU64U64": ([vp, vp, u64, i32, i32, vp, sz, vp], st),
    "gprtcuSortConfigCount": ([], i32),
    "gprtcuSortConfigAt": ([i32, vp], st),
    "gprtcuSortGetConfig": ([i32, i32, vp], st),
    "gprtcuSortSetConfig": ([i32, i32, vp], st),
    "gprtcuSortWithConfig": ([vp, vp, u64, i32, i32, i32, i32, vp, vp, sz, vp], st),
    "gprtcuSortAutotune": ([i32, i32, u64, i32, vp, i32, vp, vp, vp], st),
    "gprtcuLbvhScratchSize": ([u32], sz),
    "gprtcuLbvhBuildTriangles": ([vp, vp, u32, i32, vp, vp, sz, vp], st),
    "gprtcuLbvhBuildPoints": ([vp, u32, i32, vp, vp, sz, vp], st),
    "gprtcuLbvhBuildEdges": ([vp, vp, u32, i32, vp, vp, sz, vp], st),
    "gprtcuLbvhRefitTriangles": ([vp, vp, vp, u32, vp, vp, sz, vp], st),
    "gprtcuSphereBounds": ([vp, u32, vp, vp], st),
    "gprtcuLssBounds": ([vp, vp, u32, i32, i32, vp, vp], st),
    "gprtcuLbvhBuildBoxes": ([vp, u32, i32, vp, vp, sz, vp], st),
    "gprtcuTraceSpheres": ([vp, vp, vp, u64, i32, i32, vp, vp, vp, sz, vp], st),
    "gprtcuTraceLss": ([vp, vp, vp, i32, i32, vp, u64, i32, i32, vp, vp, vp, sz, vp], st),
    "gprtcuSolidBounds": ([vp, vp, vp, vp], st),
    "gprtcuLocateSolidPoints": ([vp, vp, vp, u64, vp, vp, vp, sz, vp], st),
    "gprtcuInstancesPrepare": ([vp, u32, vp, u32, vp, vp, vp], st),
    "gprtcuTraceInstances": ([vp, vp, vp, vp, vp, u32, vp, u64, u32, i32, vp, vp, vp, sz, vp], st),
    "gprtcuTraceScratchSize": ([], sz),
    "gprtcuTraceClosest": ([vp, vp, u64, vp, vp, sz, vp], st),
    "gprtcuTraceAny": ([vp, vp, u64, vp, vp, sz, vp], st),
    "gprtcuBatchScratchSize": ([u32, u32], sz),
    "gprtcuBatchBuildTriangles": ([vp, vp, vp, u32, u32, i32, vp, vp, sz, vp], st),
    "gprtcuBatchTrace": ([vp, vp, vp, u32, vp, u64, i32, vp, vp, sz, vp], st),
    "gprtcuWideScratchSize": ([u32, u32], sz),
    "gprtcuWideBuild": ([vp, vp, u32, vp, vp, sz, vp], st),
    "gprtcuWideTrace": ([vp, vp, u32, vp, u64, i32, vp, vp, sz, vp], st),
    "gprtcuGenSoup": ([u64, u64, ctypes.c_float, vp, u32, ctypes.c_float, vp, vp, vp], st),
    "gprtcuGenMixture": ([u64, u32, u64, ctypes.c_float, vp, vp, vp], st),
    "gprtcuGenRays": ([u64, u64, vp, u32, vp, vp, vp], st),
    "gprtcuDebugSetSpinBudget": ([u32], None),
    "gprtcuDebugScanSkipTile": ([i64], None),
    "gprtcuDebugScanSkipStage": ([i64], None),
    "gprtcuDebugSortSkipTile": ([i64], None),
    "gprtcuDebugSortRanking": ([i32], None),
    "gprtcuDebugSortPrefetch": ([i32], None),
    "gprtcuDebugRefitSkipLeaf": ([i64], st),
    "gprtcuDebugScanImpl": ([i32], None),
}


def declare(L):
    for name, (args, res) in SIGNATURES.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = res
