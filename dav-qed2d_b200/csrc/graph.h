// graph.h -- CUDA-graph replay of the molecular-dynamics part of a trajectory.
//
// The MD integration of an HMC trajectory (every force evaluation with its
// persistent solver launch, kicks and link updates) is a fixed sequence of
// launches for fixed arguments: the same kernels with the same parameters, on
// buffers whose addresses do not change.  A GraphCache captures that sequence
// once into a CUDA graph and replays it with one cudaGraphLaunch per
// trajectory, instead of enqueuing every launch from the host.
//
// Protocol (run_graphed):
//   * the first call with a given key runs the body directly: it tunes the
//     solver schedules (host-synchronising, not capturable) and allocates the
//     workspace the body needs;
//   * the next call with the same key captures the body on a private
//     non-blocking stream (relaxed mode), instantiates the graph and launches it
//     on the caller's stream; later calls with that key only launch it;
//   * a different key (other arguments, pointers, schedule or workspace
//     generation) starts over; a capture that fails turns graphs off for this
//     owner and runs the body directly (nothing of a failed capture executed).
// The key must name everything the body bakes into its launches.  Results are
// bitwise those of direct execution: the same launches in the same order.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <cstdio>
#include <string>

#include "internal.h"

namespace qed2d {

// key builder: exact text of doubles (%a), integers and pointers
struct GraphKey {
    std::string s;
    GraphKey& d(double v) {
        char b[40];
        std::snprintf(b, sizeof b, "%a;", v);
        s += b;
        return *this;
    }
    GraphKey& i(long long v) {
        s += std::to_string(v);
        s += ';';
        return *this;
    }
    GraphKey& p(const void* v) {
        char b[24];
        std::snprintf(b, sizeof b, "%p;", v);
        s += b;
        return *this;
    }
};

// Runs body() -- which enqueues on `stream` (a reference to the owner's stream
// field, temporarily pointed at the capture stream while capturing).
template <class Body>
int run_graphed(GraphCache& g, cudaStream_t& stream, const std::string& key, Body body) {
    if (!g.on) return body();
    if (g.exec && g.key == key) {
        QCHECK(cudaGraphLaunch(g.exec, stream));
        count_launch((int)g.nlaunch);
        g.replays++;
        return QED2D_OK;
    }
    if (g.warm != key) {   // first run with these arguments: direct
        g.drop();
        const int st = body();
        if (st == QED2D_OK) g.warm = key;
        return st;
    }
    g.drop();
    if (!g.cap && cudaStreamCreateWithFlags(&g.cap, cudaStreamNonBlocking) != cudaSuccess) {
        cudaGetLastError();
        g.on = false;
        g.failures++;
        return body();
    }
    cudaStream_t user = stream;
    const int64_t l0 = launches();
    int st = QED2D_OK;
    cudaGraph_t graph = nullptr;
    cudaError_t e = cudaStreamBeginCapture(g.cap, cudaStreamCaptureModeRelaxed);
    if (e == cudaSuccess) {
        stream = g.cap;
        st = body();
        stream = user;
        e = cudaStreamEndCapture(g.cap, &graph);
    }
    const int64_t n = launches() - l0;
    count_launch(-(int)n);   // nothing of the capture ran
    if (e == cudaSuccess && st == QED2D_OK && graph) e = cudaGraphInstantiate(&g.exec, graph, 0);
    if (graph) cudaGraphDestroy(graph);
    if (e != cudaSuccess || st != QED2D_OK || !g.exec) {
        cudaGetLastError();   // capture errors are not sticky
        g.drop();
        g.on = false;
        g.failures++;
        return body();
    }
    g.key = key;
    g.nlaunch = n;
    g.captures++;
    QCHECK(cudaGraphLaunch(g.exec, stream));
    count_launch((int)n);
    g.replays++;
    return QED2D_OK;
}

}  // namespace qed2d
