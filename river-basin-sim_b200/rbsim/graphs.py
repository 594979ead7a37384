"""CUDA graph capture of library launches, without the allocator housekeeping.

``torch.cuda.graph()`` synchronizes the device, runs Python's garbage collector
and empties torch's allocator cache before every capture. The step graphs here are
captured each time a clock or an ensemble is built, and that host work can cost
more than the steps themselves (and then re-allocating what the cache gave back).
``capture`` records what ``enqueue`` launches on a side stream directly: the
launches are the library's own kernels on raw stream handles, and no torch
allocation happens during the capture. The capture is thread-local, so another
host thread (the frame writers of ``rbsim.io`` and ``rbsim.serve``) may keep waiting
on its own copy events while a graph is recorded.
"""

from __future__ import annotations

from collections.abc import Callable

import torch


def capture(device: torch.device, enqueue: Callable[[int], None]) -> torch.cuda.CUDAGraph:
    """Capture ``enqueue(stream_handle)`` into a graph; the current stream waits for it."""
    g = torch.cuda.CUDAGraph()
    cur = torch.cuda.current_stream(device)
    side = torch.cuda.Stream(device)
    side.wait_stream(cur)
    with torch.cuda.stream(side):
        # thread-local capture: a frame-writer thread may wait on its copy events meanwhile
        g.capture_begin(capture_error_mode="thread_local")
        try:
            enqueue(side.cuda_stream)
        finally:
            g.capture_end()
    cur.wait_stream(side)
    return g
