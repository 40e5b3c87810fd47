"""Empty stand-in: the registration path never plots."""


class LineCollection:
    def __init__(self, *args, **kwargs):
        pass
