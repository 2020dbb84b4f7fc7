// Included by the reference but never called on the hot path.
#pragma once
