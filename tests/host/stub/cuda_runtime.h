// Host-only stand-in so the device physics headers compile with g++ (tests).
#pragma once
