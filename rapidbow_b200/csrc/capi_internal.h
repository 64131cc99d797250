// Internal helpers shared by the C-ABI translation units.
#pragma once
#include "rapidbow_b200.h"
#include "vocabulary.h"

#include <functional>

namespace rbw {
// The Vocabulary behind a C handle (throws kInvalidArg for a null handle).
const Vocabulary& vocabularyOf(const rbw_vocabulary* h);
// Runs f, converting exceptions to an rbw_status and the message for rbw_last_error().
int runGuarded(const std::function<void()>& f);
} // namespace rbw
