// CUDA graphs of the asynchronous device entry points (no reference
// counterpart; the reference launches each 32-step lighting chunk and waits
// for it, nh/lightmap_cuda.py:226-276).
//
// ls200_capture_begin puts the context's stream into capture mode; every
// later asynchronous call on the context (ls200_lighting_device over its time
// chunks, the march and segment device entries, ...) is recorded instead of
// run; ls200_capture_end instantiates the graph.  ls200_graph_launch replays
// it on the context's stream with one launch: the recorded kernels read and
// write the same device buffers, whose contents may change between launches.
// A call that must wait for the device (a host copy-back) is not allowed
// while capturing: CUDA reports it, the call returns an error and the
// capture is invalidated (ls200_capture_end then fails and the stream
// returns to normal).
#include "lighting.cuh"

struct ls200_graph {
    ls200_context *ctx = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    size_t nodes = 0;
};

using namespace ls200;

extern "C" ls200_status ls200_capture_begin(ls200_context *ctx) {
    return guard([&] {
        LS_REQUIRE(ctx, "NULL argument");
        std::lock_guard<std::mutex> hold(ctx->lock);
        LS_REQUIRE(ctx->stream != nullptr,
                   "graph capture needs a created stream, not the legacy default stream");
        activate(ctx);
        // Constant tables are copied before capture (a synchronous copy may
        // not run inside it).
        ensure_lighting_constants(ctx);
        LS_CUDA(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
    });
}

extern "C" ls200_status ls200_capture_end(ls200_context *ctx, ls200_graph **out) {
    return guard([&] {
        LS_REQUIRE(ctx && out, "NULL argument");
        std::lock_guard<std::mutex> hold(ctx->lock);
        activate(ctx);
        cudaGraph_t graph = nullptr;
        const cudaError_t ended = cudaStreamEndCapture(ctx->stream, &graph);
        if (ended != cudaSuccess) {
            if (graph) cudaGraphDestroy(graph);
            cudaGetLastError();
            throw Error(LS200_ERR_INVALID,
                        std::string("capture failed (a call inside it needed the host): ") +
                            cudaGetErrorString(ended));
        }
        auto g = new ls200_graph();
        g->ctx = ctx;
        g->graph = graph;
        try {
            LS_CUDA(cudaGraphGetNodes(graph, nullptr, &g->nodes));
            LS_CUDA(cudaGraphInstantiate(&g->exec, graph, 0));
        } catch (...) {
            cudaGraphDestroy(graph);
            delete g;
            throw;
        }
        *out = g;
    });
}

extern "C" ls200_status ls200_graph_launch(ls200_graph *g) {
    return guard([&] {
        LS_REQUIRE(g && g->exec, "NULL graph");
        std::lock_guard<std::mutex> hold(g->ctx->lock);
        activate(g->ctx);
        LS_CUDA(cudaGraphLaunch(g->exec, g->ctx->stream));
    });
}

extern "C" ls200_status ls200_graph_nodes(ls200_graph *g, int64_t *nodes) {
    return guard([&] {
        LS_REQUIRE(g && nodes, "NULL argument");
        *nodes = static_cast<int64_t>(g->nodes);
    });
}

extern "C" ls200_status ls200_graph_destroy(ls200_graph *g) {
    return guard([&] {
        if (!g) return;
        if (g->exec) cudaGraphExecDestroy(g->exec);
        if (g->graph) cudaGraphDestroy(g->graph);
        delete g;
    });
}
