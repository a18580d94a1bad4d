"""Host<->device traffic of the Python entry points (bytes), for end-to-end accounting."""
TRAFFIC = {"h2d": 0, "d2h": 0}


def reset():
    TRAFFIC["h2d"] = 0
    TRAFFIC["d2h"] = 0


def h2d(nbytes: int):
    TRAFFIC["h2d"] += int(nbytes)


def d2h(nbytes: int):
    TRAFFIC["d2h"] += int(nbytes)
