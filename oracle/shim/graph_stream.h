// Project-written empty stand-in for StreamingUtilities' graph_stream.h (not vendored with
// the reference). include/types.h includes it; the sketch / CC sources need nothing from it.
#pragma once
